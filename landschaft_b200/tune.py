"""Autotuner of the window solver (no counterpart in the reference, whose direct solver has no such choices).

For one window shape (2 (radius + buffer) + 1 cells wide), neighbourhood, edge weights and arithmetic, the
autotuner times every candidate (preconditioner, threads per window) on a sample of the caller's own windows and
installs the fastest in the library's tuning table (``lsb_tune_set``).  Calls that leave the preconditioner on
``"auto"`` and the threads per window on 0 then use it.  The table is process-wide; ``save_tuning`` and
``load_tuning`` keep it in a JSON file.

The candidates: multigrid V(1,1) or Jacobi preconditioning, with 512 or 256 threads per window (one window per
CTA, one persistent CTA per SM) or 128 (one window per CTA, four CTAs per SM: for small windows; a window too large
for a quarter of the SM's shared memory runs on 256).  Timing is the device time of the window kernels (CUDA events
around them), the best of ``repeats`` runs after one warm-up run, on a centred crop of the rasters holding about
``windows`` targets.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from . import _native as N
from .omni import EDGE_WEIGHTS, PRECONDITIONERS, active_blocks, make_params, run_device

CANDIDATES = (("mg", 512), ("mg", 256), ("mg", 128), ("jacobi", 512), ("jacobi", 256), ("jacobi", 128))

_TABLE: dict[tuple, dict] = {}  # mirror of the library's table: key -> entry


def _key(window, four, edge_weights, solver):
    return (int(window), bool(four), edge_weights, solver)


def _install(entry):
    lib = N.load()
    prec = N.PREC_FP64 if entry["solver"] == "fp64" else N.PREC_FP32_REFINE
    rc = lib.lsb_tune_set(entry["window"], int(entry["four_neighbors"]), EDGE_WEIGHTS.index(entry["edge_weights"]),
                          prec, PRECONDITIONERS.index(entry["preconditioner"]), entry["threads_per_window"])
    if rc:
        raise ValueError(f"invalid tuning entry {entry}")
    _TABLE[_key(entry["window"], entry["four_neighbors"], entry["edge_weights"], entry["solver"])] = entry


def _crop(r, s, block_size, windows):
    """A centred square crop of the rasters with about `windows` targets (the whole map if it has fewer)."""
    ny, nx = r.shape
    total = int(active_blocks(s, block_size).sum())
    if total <= windows:
        return r, s, total
    # targets scale with the area: start from the map's share, then grow until there are enough
    side = max(2 * block_size, int(min(ny, nx) * np.sqrt(windows / total)))
    while True:
        y0, x0 = (ny - side) // 2, (nx - side) // 2
        rc = np.ascontiguousarray(r[y0:y0 + side, x0:x0 + side])
        sc = np.ascontiguousarray(s[y0:y0 + side, x0:x0 + side])
        n = int(active_blocks(sc, block_size).sum())
        if n >= windows or side >= min(ny, nx):
            return rc, sc, n
        side = min(min(ny, nx), int(side * 1.2) + block_size)


def autotune(resistance, source, radius, *, buffer=0, block_size=1, four_neighbors=False, edge_weights="average",
             solver="fp32-refine", resistance_is_conductance=False, tol=1e-12, windows=1024, candidates=CANDIDATES,
             repeats=2, install=True, device=None):
    """Time the candidates on a sample of these rasters' windows; install and return the fastest.

    ``resistance`` and ``source`` are numpy rasters or tensors (NaN = NoData; sources as the solver takes them).
    Returns a dict with the chosen ``preconditioner`` and ``threads_per_window``, the window width, the sample's
    window count and every candidate's window-kernel time in milliseconds (None where the candidate failed).
    """
    import torch

    def host(a):
        if isinstance(a, torch.Tensor):
            return a.detach().to("cpu", torch.float64).numpy()
        return np.asarray(a, dtype=np.float64)

    r, s = host(resistance), host(source)
    rc, sc, n = _crop(r, s, int(block_size), int(windows))
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    rt, st = torch.from_numpy(rc).to(dev), torch.from_numpy(sc).to(dev)
    times = {}
    for pc, nt in candidates:
        p = make_params(radius, buffer, block_size, four_neighbors=four_neighbors,
                        resistance_is_conductance=resistance_is_conductance, edge_weights=edge_weights,
                        solver=solver, preconditioner=pc, tol=tol, threads_per_window=nt, use_graph=False,
                        correct_artifacts=False)
        try:
            run_device(rt, st, p)
            best = min(run_device(rt, st, p, time_windows=True)[2] for _ in range(max(1, repeats)))
            times[f"{pc}/{nt}"] = best * 1e3
        except N.NativeError:
            times[f"{pc}/{nt}"] = None
    ok = {k: v for k, v in times.items() if v is not None}
    if not ok:
        raise RuntimeError(f"no candidate solved the sample: {times}")
    choice = min(ok, key=ok.get)
    pc, nt = choice.split("/")
    entry = {"window": 2 * (int(radius) + int(buffer)) + 1, "four_neighbors": bool(four_neighbors),
             "edge_weights": edge_weights, "solver": solver, "preconditioner": pc, "threads_per_window": int(nt),
             "sample_windows": n, "window_ms": times}
    if install:
        _install(entry)
    return entry


def tuning_table():
    """The entries installed by this process (autotune or load_tuning)."""
    return [dict(e) for e in _TABLE.values()]


def save_tuning(path):
    Path(path).write_text(json.dumps(tuning_table(), indent=1))


def load_tuning(path):
    """Install the entries of a file written by save_tuning; returns how many."""
    entries = json.loads(Path(path).read_text())
    for e in entries:
        _install(e)
    return len(entries)


def clear_tuning():
    N.load().lsb_tune_clear()
    _TABLE.clear()
