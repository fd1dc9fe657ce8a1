"""Benchmark of the Omniscape moving-window solve on B200 (one JSON line on rank 0).

Workload (``omni_1024``): 1024 x 1024 Gaussian-random-field resistance 10^(2g) with ~1% NoData in 3 x 3
clusters, source 1 where g < 0.3; radius 32, block 3, 8 neighbours, average-conductance edges, block-artifact
correction on; cumulative current.  A step is one full Omniscape run over the raster (every target window solved
and scattered).

* ``value``: windows/s of the FP32-CG + FP64-refinement solve with the rasters resident in HBM, device time
  (CUDA events), L2 flushed between steps, max over ranks; every rank solves its own seeded raster (weak
  scaling, no collective on the data path).
* ``e2e``: the same metric through the drop-in ``landschaft_b200.omniscape(numpy, ...)`` call: host rasters
  in, host maps out, the copies inside the timed region.
* ``fp64``: the plain FP64 Jacobi-PCG GPU path on the same workload; ``fp32_over_fp64`` their ratio.  The FP32
  solve's preconditioner and threads per window are the autotuner's choice on a sample of the map's windows.
* ``max_rel_err``: max relative error of the cumulative current over the cells above 1e-12 of the maximum,
  against the reference's own driver (oracle/_ref, FP64 direct solves) on the whole map (maps of more than 20,000
  windows: a centred crop of at least 2,000), for both GPU solvers; also FP32 against FP64.
* ``cpu_baseline``: that reference run, timed on the host cores (rank 0, N = 1).
* ``roofline``: the window kernel's algorithmic HBM bytes (32 B per window cell: resistance and source read,
  current read and written) over its event time; ``smem``: its algorithmic shared-memory bytes per CG
  iteration (84 B per unknown) over the same time.

``--impl reference`` times that CPU reference alone, each step one run over the whole map.
``--profile-run`` runs the FP32 solve once (optionally on a centred ``--crop``), for profiler captures.
``--workload advanced_4096`` times the advanced-mode batch instead (4096 independent rasters, one launch per step).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Omniscape windows/s: batched FP32+refine vs plain FP64 GPU, at <=1e-6 rel err"


def workload_config(name, r, kw):
    return {"workload": name, "raster": f"{r.shape[0]}x{r.shape[1]}", "radius": kw["radius"],
            "block_size": kw["block_size"], "buffer": kw["buffer"], "neighbours": 8, "edge_weights": "average",
            "outputs": "cum_currmap"}


SMEM_BYTES_PER_CYCLE = 128  # shared-memory bandwidth of one SM
SMS = 148


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------------------------------------------

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    """Process group plumbing: barrier and max over ranks (no collective on the data path)."""

    def __init__(self, world, backend):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------------------------

class Clocks:
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------------------------
# the CPU reference (bounded sample)
# ---------------------------------------------------------------------------------------------------------------

def run_cpu_reference(r, s, kw, threads):
    """The reference's own driver (oracle/_ref; else the C restatement) over the whole map: (seconds, windows,
    kind, cumulative current)."""
    import oracle
    kind = "reference" if oracle.REF_AVAILABLE else "port"
    t0 = time.perf_counter()
    out = oracle.core_omniscape(r, s, kw["radius"], kw["buffer"], kw["block_size"], False, False, True, False,
                                threads=threads, impl="ref" if kind == "reference" else "port")
    dt = time.perf_counter() - t0
    return dt, out["n_targets"], kind, out["current"]


SAMPLE = "the whole map, every target window (FP64 direct solves)"
FULL_MAP_WINDOWS = 20000  # larger maps: the CPU reference runs on a centred crop


def cpu_crop(r, s, kw, windows=2000):
    """A centred square crop with at least `windows` targets (grown from two block sizes)."""
    from landschaft_b200.omni import active_blocks
    ny, nx = r.shape
    bs = kw["block_size"]
    side = 2 * bs
    while True:
        y0, x0 = (ny - side) // 2, (nx - side) // 2
        rc = np.ascontiguousarray(r[y0:y0 + side, x0:x0 + side])
        sc = np.ascontiguousarray(s[y0:y0 + side, x0:x0 + side])
        n = int(active_blocks(sc, bs).sum())
        if n >= windows or side >= min(ny, nx):
            return rc, sc, f"the centred {side} x {side} crop of the map, every target window ({n}; FP64 direct solves)"
        side = min(min(ny, nx), int(side * 1.25) + bs)


# ---------------------------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------------------------

def max_rel(ours, want):
    top = np.nanmax(np.abs(want))
    m = ~np.isnan(want) & (np.abs(want) > 1e-12 * top)
    return float(np.max(np.abs(ours[m] - want[m]) / np.abs(want[m]))) if m.any() else 0.0


def patterns_match(ours, want):
    """NaN and zero cells in the same places."""
    return bool(np.array_equal(np.isnan(ours), np.isnan(want)) and np.array_equal(ours == 0, want == 0))


def time_device(lsb_om, rt, st, params, steps, warmup, flush):
    """Per-step device times (CUDA events on the caller's stream, which waits for the call's stream)."""
    import torch
    for _ in range(warmup):
        lsb_om.run_device(rt, st, params, want_stats=False)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        lsb_om.run_device(rt, st, params, want_stats=False)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    return times


def kernel_time(lsb_om, rt, st, params, flush, reps=3):
    """Duration of the window kernels alone (CUDA events on the stream they are launched on), best of reps."""
    import torch
    from landschaft_b200 import _native as N
    p = N.Params.from_buffer_copy(params)
    p.use_graph = 0
    durs = []
    stats = None
    for _ in range(reps):
        flush.zero_()
        _, stats, kt = lsb_om.run_device(rt, st, p, time_windows=True)
        durs.append(kt)
    torch.cuda.synchronize()
    return min(durs), stats


ADV_METRIC = "advanced-mode rasters/s: 4096 independent grounded raster circuits, FP32 CG + FP64 refinement"


PW_METRIC = "Circuitscape pairwise: pair solves/s (unit current between two focal nodes, node currents included)"


def bench_pairwise(args, rank, world, local, d):
    """Circuitscape's pairwise mode with current maps on a 256 x 256 raster with 24 focal points (276 pairs, every
    pair solved).  The graph is a plain grid, so the pairs run on the raster solver (as circuitscape_pairwise routes
    them): a step is one lsb_rasters call over the 276 pair rasters (unit source at the pair's destination, direct
    ground at its source), inputs resident on the device.  The node-graph kernel (lsb_graph_pairs, Jacobi CG) is
    timed beside it over the same pairs."""
    import torch
    from landschaft_b200 import circuitscape as cs, raster as RA, synthetic
    r, pm = synthetic.pairwise_256(rank)
    dev = torch.device("cuda", local)
    g = cs.habitat_conductance(np.where(np.isnan(r), cs.NODATA, r))
    graph = cs.raster_graph(g, None, False, False)
    fp = cs._points_from_map(pm)
    rows, cols = fp.cells
    nodes = graph.nodemap[rows * g.shape[1] + cols]
    k = graph.comp[nodes[0]]
    nodes = nodes[graph.comp[nodes] == k]
    members = np.flatnonzero(graph.comp == k)
    sys_ = cs.component_system(graph, members)
    dsys = cs.system_to_device(sys_, dev)
    ground = int(sys_.local[members[-1]])
    pairs = [(a, b) for a in range(len(nodes)) for b in range(a + 1, len(nodes))]
    src = torch.tensor([int(sys_.local[nodes[a]]) for a, _ in pairs], dtype=torch.int32, device=dev)
    dst = torch.tensor([int(sys_.local[nodes[b]]) for _, b in pairs], dtype=torch.int32, device=dev)
    n, nj = len(members), len(pairs)
    # the raster route: one packed batch of pair rasters
    assert cs.raster_route(graph)
    ncell = g.size
    on = np.flatnonzero(graph.nodemap >= 0)
    node_cell = np.empty(graph.n_nodes, dtype=np.int64)
    node_cell[graph.nodemap[on]] = on
    base = np.arange(nj, dtype=np.int64) * ncell
    G = torch.from_numpy(np.ascontiguousarray(g).ravel()).to(dev).repeat(nj)
    S = torch.zeros(nj * ncell, dtype=torch.float64, device=dev)
    GR = torch.zeros_like(S)
    S[torch.from_numpy(base + node_cell[[nodes[b] for _, b in pairs]]).to(dev)] = 1.0
    GR[torch.from_numpy(base + node_cell[[nodes[a] for a, _ in pairs]]).to(dev)] = np.inf
    rp = RA.raster_params(four_neighbors=False, tol=1e-12)
    shapes = [g.shape] * nj
    if args.profile_run:  # the first 96 pairs on both routes (the graph kernel's vectors, 200 MB, exceed L2)
        _, _, rst = RA.run_rasters(G[:96 * ncell], S[:96 * ncell], GR[:96 * ncell], shapes[:96], rp)
        _, _, st = cs.solve_pairs(dsys, ground, src[:96], dst[:96])
        print(json.dumps({"profile_run": "pairwise_256 (first 96 pairs)", "nodes": n,
                          "raster_cg_iterations_mean": rst.iters_total / max(rst.n_solved, 1),
                          "graph_cg_iterations_mean": st.iters_mean}), flush=True)
        d.close()
        return
    _, _, rst = RA.run_rasters(G, S, GR, shapes, rp)
    RA.run_rasters(G, S, GR, shapes, rp, want_stats=False)
    launches = int(__import__("landschaft_b200").omni.last_launch_count())  # kernels of one timed call
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        RA.run_rasters(G, S, GR, shapes, rp, want_stats=False)
    clocks = Clocks(local)
    d.barrier()
    torch.cuda.synchronize()
    clocks.start()
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        RA.run_rasters(G, S, GR, shapes, rp, want_stats=False)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    clk = clocks.stop()
    d.barrier()
    T = d.max(sum(times))
    # the node-graph kernel over the same pairs (one timed call after one untimed)
    _, _, st = cs.solve_pairs(dsys, ground, src, dst)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    cs.solve_pairs(dsys, ground, src, dst, stats=False)
    e1.record()
    torch.cuda.synchronize()
    t_graph = d.max(e0.elapsed_time(e1) / 1e3)
    # end to end: the public call from host rasters (graph, solves, maps)
    te = []
    for _ in range(max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = cs.circuitscape_pairwise(r, pm, cum_map=True, device=dev)
        te.append(time.perf_counter() - t0)
    TE = d.max(sum(te) / len(te))
    err = None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, str(Path(__file__).resolve().parent / "oracle"))
        import circuitscape_oracle as O
        G = O.raster_graph(g, None, False, False)
        mem = [v for v in range(G["n_nodes"]) if G["comp"][v] == k]
        t0 = time.perf_counter()
        loc, lu = O._component_solver(G, mem, mem[-1])
        R = np.zeros(len(pairs))
        for q, (a, b) in enumerate(pairs):
            bvec = np.zeros(len(loc))
            s_, d_ = int(nodes[a]), int(nodes[b])
            if s_ in loc:
                bvec[loc[s_]] = -1.0
            if d_ in loc:
                bvec[loc[d_]] = 1.0
            x = lu.solve(bvec)
            R[q] = (x[loc[d_]] if d_ in loc else 0.0) - (x[loc[s_]] if s_ in loc else 0.0)
        dt = time.perf_counter() - t0
        ours = np.array([res.resistances[1 + a, 1 + b] for a, b in pairs])
        err = float(np.max(np.abs(ours - R) / np.abs(R)))
        cpu = {"value": nj / dt, "unit": "pairs/s", "cores": 1, "kind": "port",
               "sample": f"the oracle: the component's sparse LU (scipy SuperLU, one thread) and all {nj} pair solves "
                         "(resistances only, no currents); the reference factorises once the same way"}
    if rank == 0:
        line = {"metric": PW_METRIC, "value": world * nj * args.steps / T, "unit": "pairs/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 CG + f64 refinement",
                "data": "synthetic (seeded Gaussian random field, 24 random focal points)",
                "config": {"workload": "pairwise_256", "nodes": n, "pairs": nj, "neighbours": 8,
                           "l2": "flushed between timed steps (256 MiB write)", "tol": 1e-12},
                "e2e": {"value": world * nj / TE, "unit": "pairs/s",
                        "h2d_bytes_per_step": int(8 * g.size + 2 * 8 * nj),
                        "d2h_bytes_per_step": int(8 * nj * len(nodes) + 2 * 8 * n),
                        "includes": "host graph build; the conductance raster and the pairs' cells in, the focal "
                                    "voltages and the summed and largest currents out; the cum map on the host"},
                "solver": "lsb_rasters (FP32 CG, multigrid, FP64 refinement to 1e-12)",
                "cg_iterations": {"mean": rst.iters_total / max(rst.n_solved, 1), "max": rst.iters_max},
                "graph_kernel": {"value": world * nj / t_graph, "unit": "pairs/s", "kernel": "lsb_graph_pairs",
                                 "cg_iterations_mean": st.iters_mean, "ctas": st.ctas,
                                 "worst_residual": st.worst_residual}, "max_rel_err_vs_oracle": err, "clocks": clk,
                "gpu_launches": launches * args.steps, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    d.close()


O2A_METRIC = "Circuitscape one-to-all: problems/s (unit current from one focal point, the others direct grounds)"


def bench_one_to_all(args, rank, world, local, d):
    """Circuitscape's one-to-all mode with current maps on the pairwise_256 raster and its 24 focal points (24
    problems).  A step is one lsb_rasters call over the 24 problem rasters (the route the package takes on a plain
    grid), inputs resident on the device; the node-graph route (lsb_graph_solve) is timed beside it."""
    import torch
    from landschaft_b200 import circuitscape as cs, raster as RA, synthetic
    r, pm = synthetic.pairwise_256(rank)
    dev = torch.device("cuda", local)
    g = cs.habitat_conductance(np.where(np.isnan(r), cs.NODATA, r))
    fp = cs._points_from_map(pm)
    rows, cols = fp.cells
    cells = rows * g.shape[1] + cols
    npnt = len(cells)
    ncell = g.size
    # problem k: unit source at point k, every other point a direct ground (all points lie in one component)
    S = torch.zeros(npnt * ncell, dtype=torch.float64, device=dev)
    GR = torch.zeros_like(S)
    for k in range(npnt):
        S[k * ncell + int(cells[k])] = 1.0
        others = torch.from_numpy(k * ncell + np.delete(cells, k)).to(dev)
        GR[others] = np.inf
    G = torch.from_numpy(np.ascontiguousarray(g).ravel()).to(dev).repeat(npnt)
    rp = RA.raster_params(four_neighbors=False, tol=1e-12)
    shapes = [g.shape] * npnt
    _, _, rst = RA.run_rasters(G, S, GR, shapes, rp)
    RA.run_rasters(G, S, GR, shapes, rp, want_stats=False)
    launches = int(__import__("landschaft_b200").omni.last_launch_count())  # kernels of one timed call
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        RA.run_rasters(G, S, GR, shapes, rp, want_stats=False)
    clocks = Clocks(local)
    d.barrier()
    torch.cuda.synchronize()
    clocks.start()
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        RA.run_rasters(G, S, GR, shapes, rp, want_stats=False)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    clk = clocks.stop()
    d.barrier()
    T = d.max(sum(times))
    # end to end through the public call, and the node-graph route over the same problems
    kw = dict(current_maps=True, device=dev)
    res = cs.circuitscape_one_to_all(r, pm, **kw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = cs.circuitscape_one_to_all(r, pm, **kw)
    TE = d.max(time.perf_counter() - t0)
    cs.circuitscape_one_to_all(r, pm, problem_solver="graph", **kw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    resg = cs.circuitscape_one_to_all(r, pm, problem_solver="graph", **kw)
    TG = d.max(time.perf_counter() - t0)
    cpu = None
    err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, str(Path(__file__).resolve().parent / "oracle"))
        import circuitscape_oracle as O
        opts = {"volt_maps": False, "cur_maps": True, "cum": True, "max": False, "focal_zero": False}
        t0 = time.perf_counter()
        want = cs._one_to_all(g, None, fp, None, None, True, False, False, opts, lambda *a: None, O.multi_advanced)
        dt = time.perf_counter() - t0
        err = float(np.max(np.abs(res.resistances[:, 1] - want.resistances[:, 1]) / np.abs(want.resistances[:, 1])))
        cpu = {"value": npnt / dt, "unit": "problems/s", "cores": 1, "kind": "port",
               "sample": f"the oracle: all {npnt} problems, each a sparse LU (scipy SuperLU, one thread) of the "
                        "component, with node currents and the cum map (the graph built with plain loops)"}
    if rank == 0:
        line = {"metric": O2A_METRIC, "value": world * npnt * args.steps / T, "unit": "problems/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 CG + f64 refinement", "data": "synthetic (the pairwise_256 raster and focal points)",
                "config": {"workload": "one_to_all_256", "cells": int(ncell), "problems": npnt, "neighbours": 8,
                           "l2": "flushed between timed steps (256 MiB write)", "tol": 1e-12},
                "solver": "lsb_rasters (FP32 CG, multigrid, FP64 refinement)",
                "cg_iterations": {"mean": rst.iters_total / max(rst.n_solved, 1), "max": rst.iters_max},
                "e2e": {"value": world * npnt / TE, "unit": "problems/s",
                        "h2d_bytes_per_step": int(2 * 8 * ncell), "d2h_bytes_per_step": int(npnt * 2 * 8 * ncell),
                        "includes": "host graph build, problem construction, all per-point current maps"},
                "graph_route_e2e": {"value": world * npnt / TG, "unit": "problems/s",
                                    "solver": "lsb_graph_solve (FP64 Jacobi CG)",
                                    "max_rel_diff_vs_raster_route": float(np.max(
                                        np.abs(resg.resistances[:, 1] - res.resistances[:, 1])
                                        / np.abs(res.resistances[:, 1])))},
                "max_rel_err_vs_oracle": err, "clocks": clk, "gpu_launches": launches * args.steps, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    d.close()


def bench_advanced(args, rank, world, local, d):
    """The advanced-mode batch: 4096 rasters of sides U{64..512}, log-uniform resistance in [1, 1000], one unit
    source and one direct ground each, 4 neighbours; a step is one launch over the whole batch."""
    import torch
    from landschaft_b200 import raster, synthetic
    shapes, g, s, gr = synthetic.advanced_packed(64 if args.profile_run else 4096, seed=rank)
    n, cells = len(shapes), g.size
    dev = torch.device("cuda", local)
    gt, st, grt = (torch.from_numpy(x).to(dev) for x in (g, s, gr))
    p = raster.raster_params(four_neighbors=True)
    if args.profile_run:
        _, _, stats = raster.run_rasters(gt, st, grt, shapes, p)
        print(json.dumps({"profile_run": "advanced_4096 (first 64 rasters)", "cells": int(cells),
                          "cg_iterations_mean": stats.iters_total / max(stats.n_solved, 1)}), flush=True)
        d.close()
        return
    _, _, stats = raster.run_rasters(gt, st, grt, shapes, p)
    launches = int(__import__("landschaft_b200").omni.last_launch_count())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        raster.run_rasters(gt, st, grt, shapes, p, want_stats=False)
    clocks = Clocks(local)
    d.barrier()
    torch.cuda.synchronize()
    clocks.start()
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        raster.run_rasters(gt, st, grt, shapes, p, want_stats=False)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    clk = clocks.stop()
    d.barrier()
    T = d.max(sum(times))
    # end to end: host rasters in (pinned), host maps out
    hosts = [torch.from_numpy(x).pin_memory() for x in (g, s, gr)]
    out_c = torch.empty(cells, dtype=torch.float64).pin_memory()
    out_v = torch.empty_like(out_c).pin_memory()
    te = []
    for _ in range(max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dg, ds, dgr = (h.to(dev, non_blocking=True) for h in hosts)
        c, v, _ = raster.run_rasters(dg, ds, dgr, shapes, p, want_stats=False)
        out_c.copy_(c, non_blocking=True)
        out_v.copy_(v, non_blocking=True)
        torch.cuda.synchronize()
        te.append(time.perf_counter() - t0)
        del dg, ds, dgr, c, v
    TE = d.max(sum(te) / len(te))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        from concurrent.futures import ThreadPoolExecutor
        kind = "reference" if oracle.REF_AVAILABLE else "port"
        offs = np.concatenate([[0], np.cumsum([a * b for a, b in shapes])])
        pick = [k for k, (a, b) in enumerate(shapes) if max(a, b) <= 128][:32]
        threads = os.cpu_count() or 1

        def one(k):
            a, b = shapes[k]
            sl = slice(offs[k], offs[k + 1])
            arr = [x[sl].reshape(a, b) for x in (g, s, gr)]
            if kind == "reference":
                return oracle.ref_advanced(*arr, four=True, threads=1)
            return oracle.advanced(*arr, four=True)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(one, pick))
        dt = time.perf_counter() - t0
        sc = sum(shapes[k][0] * shapes[k][1] for k in pick)
        cpu = {"value": len(pick) / dt, "unit": "rasters/s", "cells_per_s": sc / dt, "cores": threads, "kind": kind,
               "sample": f"{len(pick)} rasters of the batch with sides <= 128 ({sc} cells), one per host thread; "
                         "the batch's mean raster has 83,000 cells, so compare cells/s"}
    if rank == 0:
        line = {"metric": ADV_METRIC, "value": world * n * args.steps / T, "unit": "rasters/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 CG + f64 refinement",
                "data": "synthetic (seeded log-uniform resistance per raster)",
                "config": {"workload": "advanced_4096", "rasters": n, "cells": int(cells), "sides": "U{64..512}",
                           "neighbours": 4, "l2": "flushed between timed steps (256 MiB write)", "tol": 1e-12},
                "cells_per_s": world * cells * args.steps / T,
                "e2e": {"value": world * n / TE, "unit": "rasters/s", "h2d_bytes_per_step": int(3 * 8 * cells),
                        "d2h_bytes_per_step": int(2 * 8 * cells)},
                "cg_iterations": {"mean": stats.iters_total / max(stats.n_solved, 1), "max": stats.iters_max},
                "failed": int(stats.n_failed), "clocks": clk, "gpu_launches": launches * args.steps,
                "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    d.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--workload", default="omni_1024")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--crop", type=int, default=0, help="centred square crop of the workload (profile runs)")
    ap.add_argument("--profile-run", action="store_true", help="one FP32 solve of the workload and exit")
    args = ap.parse_args()
    rank, world, local = dist_env()
    from landschaft_b200 import synthetic

    if args.impl == "reference":
        if rank != 0:
            return
        r, s, kw = synthetic.omni_1024(0)
        threads = os.cpu_count() or 1
        times = []
        kind = None
        for i in range(args.warmup + args.steps):
            dt, n, kind, _ = run_cpu_reference(r, s, kw, threads)
            if i >= args.warmup:
                times.append(dt)
        v = n / statistics.mean(times)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "windows/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Gaussian random field; no dataset is published for this path)",
                "config": {**workload_config("omni_1024", r, kw), "precision": "fp64 direct (CPU)"},
                "cpu_baseline": {"value": v, "unit": "windows/s", "cores": threads, "kind": kind, "sample": SAMPLE},
                "e2e": {"value": v, "unit": "windows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    d = Dist(world, "nccl")
    import landschaft_b200 as lsb
    from landschaft_b200 import omni as lsb_om

    if args.workload == "advanced_4096":
        return bench_advanced(args, rank, world, local, d)
    if args.workload == "pairwise_256":
        return bench_pairwise(args, rank, world, local, d)
    if args.workload == "one_to_all_256":
        return bench_one_to_all(args, rank, world, local, d)
    r, s, kw = synthetic.WORKLOADS[args.workload](rank)
    if args.crop:
        y0, x0 = (r.shape[0] - args.crop) // 2, (r.shape[1] - args.crop) // 2
        r = np.ascontiguousarray(r[y0:y0 + args.crop, x0:x0 + args.crop])
        s = np.ascontiguousarray(s[y0:y0 + args.crop, x0:x0 + args.crop])
    dev = torch.device("cuda", local)
    rt = torch.from_numpy(r).to(dev)
    st = torch.from_numpy(s).to(dev)
    p32 = lsb_om.make_params(kw["radius"], kw["buffer"], kw["block_size"], solver="fp32-refine")
    p64 = lsb_om.make_params(kw["radius"], kw["buffer"], kw["block_size"], solver="fp64", preconditioner="jacobi")
    if args.profile_run:
        p = lsb_om.make_params(kw["radius"], kw["buffer"], kw["block_size"], solver="fp32-refine", use_graph=False)
        _, stats = lsb_om.run_device(rt, st, p)
        torch.cuda.synchronize()
        print(json.dumps({"profile_run": args.workload, "crop": args.crop, "windows": int(stats.n_targets),
                          "cg_iterations_mean": stats.iters_total / max(stats.n_solved, 1)}), flush=True)
        d.close()
        return
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MiB > 126 MB L2
    # the autotuner picks the FP32 solve's preconditioner and threads per window on a sample of the windows
    # (outside the timed region); p32 leaves both on auto
    tune = lsb.autotune(r, s, kw["radius"], buffer=kw["buffer"], block_size=kw["block_size"])
    # correctness and counts (outside the timed region)
    out32, stats32 = lsb_om.run_device(rt, st, p32)
    c32 = out32["current"].cpu().numpy()
    out64, stats64 = lsb_om.run_device(rt, st, p64)
    c64 = out64["current"].cpu().numpy()
    n_windows = int(stats32.n_targets)
    err = {"fp32_vs_fp64": max_rel(c32, c64)}
    lsb_om.run_device(rt, st, p32)
    launches = int(lsb_om.last_launch_count())

    # device-resident timing, FP32 + refinement
    clocks = Clocks(local)
    d.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t32 = time_device(lsb_om, rt, st, p32, args.steps, args.warmup, flush)
    clk = clocks.stop()
    d.barrier()
    torch.cuda.synchronize()
    T32 = d.max(sum(t32))
    value = world * n_windows * args.steps / T32
    # plain FP64
    t64 = time_device(lsb_om, rt, st, p64, max(1, min(args.steps, 3)), 1, flush)
    T64 = d.max(sum(t64) / len(t64))
    fp64_value = world * n_windows / T64
    # e2e through the drop-in call (host numpy in, host maps out)
    for _ in range(max(1, args.warmup)):
        lsb.omniscape(r, kw["radius"], source=s, block_size=kw["block_size"], mask_nodata=False)
    torch.cuda.synchronize()
    d.barrier()
    te = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        lsb.omniscape(r, kw["radius"], source=s, block_size=kw["block_size"], mask_nodata=False)
        te.append(time.perf_counter() - t0)
    TE = d.max(sum(te))
    e2e = world * n_windows * args.steps / TE
    # window-kernel time and roofline (rank-local)
    ktime, kstats = kernel_time(lsb_om, rt, st, p32, flush)
    active = lsb_om.active_blocks(s, kw["block_size"])
    assert int(active.sum()) == n_windows
    cells = lsb_om.window_cells(r.shape, {**kw, "active": active})  # sum over targets of the window box cells
    hbm_bytes = cells * 32.0  # per window cell: resistance 8 + source 8 read, current 8 read + 8 written
    peak, peak_kind = peaks()
    achieved = hbm_bytes / ktime / 1e9
    prof = ROOT / "profiles" / "k_windows_omni_1024_traffic.json"
    traffic = (json.loads(prof.read_text())["dram_bytes_per_launch"]
               if prof.exists() and not args.crop and args.workload == "omni_1024" else None)
    smem_bytes = kstats.unknown_iters * 84.0  # per unknown and CG iteration (FP32, 8 neighbours)
    smem_peak = SMEM_BYTES_PER_CYCLE * SMS * (clk["sm_mhz"] or 1965.0) * 1e6 / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        if n_windows <= FULL_MAP_WINDOWS:
            rs, ss, sample, g32, g64 = r, s, SAMPLE, c32, c64
        else:
            rs, ss, sample = cpu_crop(r, s, kw)
            rts, sts = torch.from_numpy(rs).to(dev), torch.from_numpy(ss).to(dev)
            g32 = lsb_om.run_device(rts, sts, p32)[0]["current"].cpu().numpy()
            g64 = lsb_om.run_device(rts, sts, p64)[0]["current"].cpu().numpy()
        dt, n, kind, cref = run_cpu_reference(rs, ss, kw, threads)
        cpu = {"value": n / dt, "unit": "windows/s", "cores": threads, "kind": kind, "sample": sample}
        err["fp32_vs_reference"] = max_rel(g32, cref)
        err["fp64_vs_reference"] = max_rel(g64, cref)
        err["nan_and_zero_patterns_match"] = patterns_match(g32, cref) and patterns_match(g64, cref)
        err["reference_sample"] = sample
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "windows/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * T32 / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 CG + f64 refinement",
                "data": "synthetic (seeded Gaussian random field per rank; no dataset is published for this path)",
                "config": {**workload_config(args.workload, r, kw), "windows_per_rank": n_windows, "parallelism": f"{world} independent rasters",
                           "l2": "flushed between timed steps (256 MiB write)", "tol": 1e-12,
                           "autotuned": {"preconditioner": tune["preconditioner"],
                                         "threads_per_window": tune["threads_per_window"],
                                         "sample_windows": tune["sample_windows"], "window_ms": tune["window_ms"]}},
                "e2e": {"value": e2e, "unit": "windows/s", "h2d_bytes_per_step": int(r.nbytes + s.nbytes),
                        "d2h_bytes_per_step": int(r.nbytes)},
                "fp64": {"value": fp64_value, "unit": "windows/s", "preconditioner": "jacobi",
                         "ms_per_step": 1e3 * T64},
                "fp32_over_fp64": value / fp64_value,
                "max_rel_err": err,
                "cg_iterations": {"fp32_mean": stats32.iters_total / max(stats32.n_solved, 1),
                                  "fp32_max": stats32.iters_max, "refine_max": stats32.refine_max,
                                  "fp64_mean": stats64.iters_total / max(stats64.n_solved, 1),
                                  "fp64_max": stats64.iters_max},
                "cells_per_s": world * cells * args.steps / T32,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "kernel": "k_windows", "kernel_ms": ktime * 1e3,
                             "note": "algorithmic HBM bytes (32 B per window cell) over the window kernel's "
                                     "event time; the solve itself runs out of shared memory"},
                "smem": {"achieved": smem_bytes / ktime / 1e9, "peak": smem_peak, "unit": "GB/s",
                         "frac": smem_bytes / ktime / 1e9 / smem_peak,
                         "note": "84 B per unknown and CG iteration over the window kernel's event time; peak = "
                                 "128 B/cycle/SM x 148 SMs x the median SM clock (nominal)"},
                "clocks": clk, "gpu_launches": launches * args.steps, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    d.close()


if __name__ == "__main__":
    main()
