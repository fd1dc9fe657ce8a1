"""Omniscape moving-window connectivity on one B200: the drop-in for ``ls.omniscape``.

Mirrors ``src/landschaft/circuit/omniscape.py`` of landschaft (argument names,
defaults, validation, warnings, preprocessing and outputs); the native call
``circuit_omniscape`` (``src/cpp/circuit/python.cpp:90-137``) is replaced by
the C ABI of ``liblsb_omni.so`` (``include/lsb_omniscape.h``), which solves
every window on the GPU.
"""

from __future__ import annotations

import ctypes as C
import threading
import warnings

import numpy as np

from . import _native as N

COMPARISONS = ("within", "equal")
COMPARE_TO_FUTURE = ("none", "1", "2", "both")
PRECISIONS = ("double", "single")
SOLVERS = ("fp32-refine", "fp64")
PRECONDITIONERS = ("auto", "jacobi", "mg")
EDGE_WEIGHTS = ("average", "series")
OUTPUTS = ("cum_currmap", "flow_potential", "normalized_cum_currmap")


# ---------------------------------------------------------------------------------------------------------------
# Preprocessing (omniscape.py:46-189, advanced.py:34-54)
# ---------------------------------------------------------------------------------------------------------------

def _to_int(value, name: str) -> int:
    """Omniscape parses Int64(round(parse(Float64, value))): halves go to even, as Python's round."""
    v = float(value)
    if not np.isfinite(v):
        raise ValueError(f"{name} must be finite")
    return int(round(v))


def _grid(values, name: str):
    """A raster (array, masked array, DataArray or CPU/GPU tensor) as float64 with NaN for NoData, and its DataArray."""
    like = None
    try:
        import torch
        if isinstance(values, torch.Tensor):
            values = values.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    if hasattr(values, "dims") and hasattr(values, "values"):  # an xarray.DataArray
        da = values.squeeze(drop=True) if "band" in values.dims else values
        v = np.array(da.values, dtype=np.float64)
        nodata = da.rio.nodata if hasattr(da, "rio") else None
        if nodata is not None and not np.isnan(nodata):
            v[v == nodata] = np.nan
        like = da
    elif isinstance(values, np.ndarray) and not isinstance(values, np.ma.MaskedArray):
        v = np.asarray(values, dtype=np.float64)  # no copy for float64: the callers only read it
    else:
        v = np.array(np.ma.filled(np.ma.asarray(values, dtype=np.float64), np.nan), dtype=np.float64)
    if v.ndim != 2:
        raise ValueError(f"the {name} must be a 2-D raster")
    return np.ascontiguousarray(v), like


def read_reclass_table(path) -> np.ndarray:
    """Read an Omniscape reclass table: two whitespace-separated columns (value, new value); ``missing`` = NoData."""
    rows = []
    with open(path, encoding="utf-8") as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if len(parts) != 2:
                raise ValueError(f"reclass table lines need two columns: {line.strip()!r}")
            rows.append([np.nan if p.strip('"') == "missing" else float(p) for p in parts])
    return np.array(rows, dtype=np.float64).reshape(-1, 2)


def _reclass_table(table) -> np.ndarray:
    if isinstance(table, (str, bytes)) or hasattr(table, "__fspath__"):
        return read_reclass_table(table)
    if isinstance(table, dict):
        table = [[k, np.nan if v is None else v] for k, v in table.items()]
    t = np.array(table, dtype=np.float64)
    if t.ndim != 2 or t.shape[1] != 2:
        raise ValueError("reclass_table must have two columns (value, new value)")
    return t


def reclassify(resistance: np.ndarray, table) -> np.ndarray:
    """Omniscape's ``reclassify_resistance!``: each row (value, new value) matched against the original values."""
    t = _reclass_table(table)
    out = resistance.copy()
    for old, new in t:
        out[resistance == old] = new
    return out


def source_from_resistance(resistance, *, r_cutoff: float = np.inf, resistance_is_conductance: bool = False,
                           reclass_table=None):
    """Omniscape's ``source_from_resistance``: 1 / resistance (or the conductance), 0 below 1 / r_cutoff and on NoData."""
    r, like = _grid(resistance, "resistance")
    if reclass_table is not None:
        r = reclassify(r, reclass_table)
    with np.errstate(divide="ignore"):
        s = r if resistance_is_conductance else 1 / r
    s = np.where(np.isnan(s) | (s < 1 / float(r_cutoff)), 0.0, s)
    if like is None:
        return s
    out = like.copy(data=s)
    out.name = "source"
    return out


def _condition(value, shape, name, dtype):
    if value is None:
        return None
    v, _ = _grid(value, name)
    if v.shape != shape:
        raise ValueError(f"{name} must have the resistance's shape")
    if dtype is np.float32:
        v = v.astype(np.float32).astype(np.float64)
    return np.ascontiguousarray(v)


# ---------------------------------------------------------------------------------------------------------------
# Results
# ---------------------------------------------------------------------------------------------------------------

class Variable:
    """A map of a :class:`Dataset` (the part of ``xarray.DataArray`` the results need)."""

    def __init__(self, name, values):
        self.name = name
        self.values = values
        self.dims = ("y", "x")

    @property
    def shape(self):
        return self.values.shape

    def __array__(self, dtype=None, copy=None):
        return np.asarray(self.values, dtype=dtype)

    def __getitem__(self, idx):
        return self.values[idx]

    def __repr__(self):
        return f"<Variable {self.name} {self.values.shape} {self.values.dtype}>"


class Dataset:
    """The maps of a run with their ``attrs``, shaped like ``xarray.Dataset`` (used when xarray is absent)."""

    def __init__(self, data: dict, attrs: dict):
        self._vars = {k: Variable(k, v) for k, v in data.items()}
        self.attrs = attrs

    @property
    def data_vars(self):
        return list(self._vars)

    def __getitem__(self, key):
        return self._vars[key]

    def __contains__(self, key):
        return key in self._vars

    def __setitem__(self, key, value):
        """``ds[name] = values`` or ``ds[name] = (dims, values)``, as xarray takes a new map."""
        values = value[1] if isinstance(value, tuple) else value
        self._vars[key] = Variable(key, np.asarray(values))

    def __iter__(self):
        return iter(self._vars)

    def keys(self):
        return self._vars.keys()

    def __getattr__(self, key):
        v = self.__dict__.get("_vars", {})
        if key in v:
            return v[key]
        raise AttributeError(key)

    def __repr__(self):
        return f"<Dataset {self.data_vars} attrs={self.attrs}>"


def _dataset(data, attrs, like):
    order = [k for k in OUTPUTS if k in data]
    try:
        import xarray as xr
    except ImportError:
        return Dataset({k: data[k] for k in order}, attrs)
    if like is None:
        return xr.Dataset({k: (("y", "x"), data[k]) for k in order}, attrs=attrs)
    return xr.Dataset({k: like.copy(data=data[k]).rename(k) for k in order}, attrs=attrs)


# ---------------------------------------------------------------------------------------------------------------
# The device call
# ---------------------------------------------------------------------------------------------------------------

class _DeviceState:
    """Per-device workspace (grown on demand) and a side stream for the calls."""

    def __init__(self, device):
        import torch
        self.device = device
        self.ws = None
        self.stream = torch.cuda.Stream(device=device)
        self.lock = threading.Lock()

    def workspace(self, nbytes):
        import torch
        if self.ws is None or self.ws.numel() < nbytes:
            self.ws = None
            self.ws = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=self.device)
        return self.ws


_states: dict = {}


def _state(device):
    key = str(device)
    if key not in _states:
        _states[key] = _DeviceState(device)
    return _states[key]


def _device(device=None):
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("landschaft_b200 needs a CUDA device (B200, sm_100a); none is available")
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise ValueError("device must be a CUDA device")
    return d if d.index is not None else torch.device("cuda", torch.cuda.current_device())


def make_params(radius, buffer=0, block_size=1, four_neighbors=False, resistance_is_conductance=False,
                correct_artifacts=True, flow_potential=False, edge_weights="average", solver="fp32-refine",
                preconditioner="auto", tol=1e-12, max_iter=20000, threads_per_window=0, use_graph=True,
                mask_nodata=False, memory_limit=0.0, conditions=None) -> N.Params:
    """The C-ABI parameter struct (conditions: dict of device tensors as the reference's binding takes them)."""
    if solver not in SOLVERS:
        raise ValueError(f"solver must be one of {SOLVERS}")
    if preconditioner not in PRECONDITIONERS:
        raise ValueError(f"preconditioner must be one of {PRECONDITIONERS}")
    if edge_weights not in EDGE_WEIGHTS:
        raise ValueError(f"edge_weights must be one of {EDGE_WEIGHTS}")
    p = N.default_params()
    p.radius, p.buffer, p.block_size = int(radius), int(buffer), int(block_size)
    p.four_neighbors = int(bool(four_neighbors))
    p.resistance_is_conductance = int(bool(resistance_is_conductance))
    p.correct_artifacts = int(bool(correct_artifacts))
    p.flow_potential = int(bool(flow_potential))
    p.edge_weights = EDGE_WEIGHTS.index(edge_weights)
    p.precision = N.PREC_FP64 if solver == "fp64" else N.PREC_FP32_REFINE
    p.preconditioner = PRECONDITIONERS.index(preconditioner)
    p.tol = float(tol)
    p.max_iter = int(max_iter)
    p.threads_per_window = int(threads_per_window)
    p.use_graph = int(bool(use_graph))
    p.mask_nodata = int(bool(mask_nodata))
    p.memory_limit = float(memory_limit or 0.0)
    if conditions:
        for k, field in ((1, "condition1"), (2, "condition2")):
            c = conditions.get(f"condition{k}")
            if c is None:
                continue
            cd = getattr(p, field)
            cd.present = c.data_ptr()
            f = conditions.get(f"condition{k}_future")
            cd.future = f.data_ptr() if f is not None else None
            cd.equal = int(conditions[f"comparison{k}"] == "equal")
            cd.lower = float(conditions[f"condition{k}_lower"])
            cd.upper = float(conditions[f"condition{k}_upper"])
    return p


def run_device(r, s, params: N.Params, *, normalized=False, out=None, want_stats=True, time_windows=False):
    """One call of ``lsb_omniscape`` on device tensors (float64, contiguous, same device).

    Returns ``(outputs, stats)``: outputs is a dict of device tensors ``current``
    and, with the flow potential, ``flow_potential`` (and ``normalized``).  The
    work runs on a side stream ordered after the caller's current stream; the
    caller's stream waits for it.  ``want_stats=False`` returns without waiting
    (stats is then None and device-side solver failures are not reported);
    ``time_windows=True`` (calls without a graph) also returns the device time
    of the window kernels in seconds.
    """
    import torch
    lib = N.load()
    if r.dtype != torch.float64 or s.dtype != torch.float64 or not r.is_cuda or r.device != s.device:
        raise ValueError("resistance and source must be float64 tensors on one CUDA device")
    r = r.contiguous()
    s = s.contiguous()
    ny, nx = r.shape
    st = _state(r.device)
    with st.lock:
        nbytes = C.c_size_t(0)
        err = C.create_string_buffer(1024)
        rc = lib.lsb_omniscape_workspace_size(nx, ny, C.byref(params), C.byref(nbytes))
        if rc:
            N.check(rc, C.create_string_buffer(b"invalid parameters"))
        ws = st.workspace(nbytes.value)
        if out is None:
            out = {"current": torch.empty((ny, nx), dtype=torch.float64, device=r.device)}
            if params.flow_potential:
                out["flow_potential"] = torch.empty_like(out["current"])
            if normalized:
                out["normalized"] = torch.empty_like(out["current"])
        stats = N.Stats() if (want_stats or time_windows) else None
        cur = torch.cuda.current_stream(r.device)
        st.stream.wait_stream(cur)
        if time_windows:
            lib.lsb_time_window_kernels(1)
        try:
            rc = lib.lsb_omniscape(r.data_ptr(), s.data_ptr(), nx, ny, C.byref(params), out["current"].data_ptr(),
                                   out["flow_potential"].data_ptr() if "flow_potential" in out else None,
                                   out["normalized"].data_ptr() if "normalized" in out else None, ws.data_ptr(),
                                   ws.numel(), C.byref(stats) if stats is not None else None, err, len(err),
                                   st.stream.cuda_stream)
        finally:
            if time_windows:
                lib.lsb_time_window_kernels(0)
        cur.wait_stream(st.stream)
        N.check(rc, err)
        if time_windows:
            return out, stats, stats.window_ms / 1e3
        return out, stats


def _fingerprint(r, s, params: N.Params) -> str:
    """Identifies a run for its checkpoint: the rasters and every parameter but the streaming fields."""
    import hashlib
    p = N.Params.from_buffer_copy(params)
    p.accumulate, p.target_begin, p.target_end, p.use_graph = 0, 0, 0, 0
    p.condition1.present = p.condition1.future = p.condition2.present = p.condition2.future = None
    h = hashlib.sha1(bytes(p))
    for t in (r, s):
        h.update(t.detach().cpu().numpy().tobytes())
    return h.hexdigest()


def run_device_streamed(r, s, params: N.Params, *, chunk_windows: int, checkpoint=None, normalized=False,
                        max_chunks=None):
    """``run_device`` in consecutive ranges of ``chunk_windows`` targets, each continuing the previous one's maps
    (bitwise the maps of one call), with a checkpoint after every range.

    ``checkpoint``: an ``.npz`` file; when it exists and belongs to the same rasters and parameters, the run resumes
    after its last range (a finished run's file returns its maps at once).  ``max_chunks``: stop after that many
    ranges (the checkpoint then holds the partial maps; the returned stats are None).  Returns
    ``(outputs, stats)`` as ``run_device``, the stats summed over the ranges.
    """
    import os
    from pathlib import Path
    import torch
    ny, nx = r.shape
    total = int(active_blocks(s.detach().cpu().numpy(), params.block_size).sum())
    key = _fingerprint(r, s, params)
    out = {"current": torch.zeros((ny, nx), dtype=torch.float64, device=r.device)}
    if params.flow_potential:
        out["flow_potential"] = torch.zeros_like(out["current"])
    if normalized:
        out["normalized"] = torch.zeros_like(out["current"])
    fields = ("n_solved", "n_failed", "iters_total", "iters_max", "refine_max", "worst_residual", "unknown_iters")
    agg = dict.fromkeys(fields, 0)
    begin, done = 0, False
    ck = Path(checkpoint) if checkpoint is not None else None
    if ck is not None and ck.exists():
        z = np.load(ck)
        if str(z["key"]) != key:
            raise ValueError(f"the checkpoint {ck} belongs to another run (other rasters or parameters)")
        for name, t in out.items():
            if name in z.files:
                t.copy_(torch.from_numpy(z[name]))
        begin, done = int(z["next_target"]), bool(z["done"])
        agg.update({k: z[k].item() for k in fields})

    def save(finished):
        if ck is None:
            return
        tmp = ck.with_name(ck.name + ".tmp.npz")
        np.savez(tmp, key=key, next_target=begin, done=finished, **{k: v.cpu().numpy() for k, v in out.items()},
                 **{k: np.array(v) for k, v in agg.items()})
        os.replace(tmp, ck)

    p = N.Params.from_buffer_copy(params)
    p.use_graph = 0
    p.accumulate = 1
    chunks = 0
    while not done:
        end = begin + max(int(chunk_windows), 1)
        last = end >= total
        p.target_begin = begin
        p.target_end = 0 if last else end
        _, st = run_device(r, s, p, normalized=normalized and last, out=out)
        for k in ("n_solved", "n_failed", "iters_total", "unknown_iters"):
            agg[k] += getattr(st, k)
        for k in ("iters_max", "refine_max", "worst_residual"):
            agg[k] = max(agg[k], getattr(st, k))
        begin, done = (total if last else end), last
        chunks += 1
        save(done)
        if not done and max_chunks is not None and chunks >= max_chunks:
            return out, None
    stats = N.Stats()
    stats.n_targets = total
    for k, v in agg.items():
        setattr(stats, k, v)
    return out, stats


def last_launch_count() -> int:
    """Kernels the last call on this thread launched (a graph replay: the graph's kernel nodes)."""
    return int(N.load().lsb_last_launch_count())


def window_cells(shape, kw) -> int:
    """Sum over the targets of a run of the cells of their window boxes; ``kw['active']`` (lattice mask, x outer,
    y inner) selects the targets, else every block centre counts."""
    ny, nx = shape
    D = kw["radius"] + kw.get("buffer", 0)
    bs = kw.get("block_size", 1)
    br = (bs - 1) // 2
    xs = np.arange(br, nx - br, bs)
    ys = np.arange(br, ny - br, bs)
    active = kw.get("active")
    hx = np.minimum(xs + D, nx - 1) - np.maximum(xs - D, 0) + 1
    hy = np.minimum(ys + D, ny - 1) - np.maximum(ys - D, 0) + 1
    cells = np.outer(hx, hy)  # lattice order: x outer, y inner
    if active is not None:
        cells = cells * active
    return int(cells.sum())


def active_blocks(source, block_size) -> np.ndarray:
    """Lattice mask (x outer, y inner) of the blocks whose source sum is > 0 (NaN counted as 0)."""
    s = np.nan_to_num(np.asarray(source, dtype=np.float64), nan=0.0)
    ny, nx = s.shape
    bs = int(block_size)
    br = (bs - 1) // 2
    nbx = (nx - 2 * br - 1) // bs + 1 if nx - 2 * br > 0 else 0
    nby = (ny - 2 * br - 1) // bs + 1 if ny - 2 * br > 0 else 0
    sums = np.zeros((nbx, nby))
    for dx in range(-br, br + 1):
        for dy in range(-br, br + 1):
            sums += s[br + dy: br + dy + bs * nby: bs, br + dx: br + dx + bs * nbx: bs][:nby, :nbx].T
    return sums > 0


def omniscape_correction(radius, buffer, block_size, four_neighbors=False, nx=1000, ny=1000, *,
                         edge_weights="average", device=None):
    """Omniscape's block-artifact correction factors, ``(2 (radius + buffer) + 1)`` squared (computed on the GPU).

    The counterpart of ``circuit_omniscape_correction`` (python.cpp:139-153).
    """
    import torch
    dev = _device(device)
    lib = N.load()
    radius, buffer, block_size = int(radius), int(buffer), int(block_size)
    w = 2 * (radius + buffer) + 1
    corr = torch.empty((w, w), dtype=torch.float64, device=dev)
    p = make_params(radius, buffer, block_size, four_neighbors, solver="fp64", preconditioner="jacobi")
    nbytes = C.c_size_t(0)
    rc = lib.lsb_omniscape_workspace_size(1, 1, C.byref(p), C.byref(nbytes))
    N.check(rc, C.create_string_buffer(b"invalid parameters"))
    need = int(nbytes.value) + 16 * w * w + 4096
    st = _state(dev)
    with st.lock:
        ws = st.workspace(need)
        err = C.create_string_buffer(1024)
        cur = torch.cuda.current_stream(dev)
        st.stream.wait_stream(cur)
        rc = lib.lsb_omniscape_correction(radius, buffer, block_size, int(bool(four_neighbors)),
                                          EDGE_WEIGHTS.index(edge_weights), int(nx), int(ny), corr.data_ptr(),
                                          ws.data_ptr(), ws.numel(), err, len(err), st.stream.cuda_stream)
        cur.wait_stream(st.stream)
        N.check(rc, err)
    return corr.cpu().numpy()


def omniscape(resistance, radius, *, source=None, block_size=1, buffer=0, source_threshold: float = 0.0,
              r_cutoff: float = np.inf, resistance_is_conductance: bool = False, four_neighbors: bool = False,
              flow_potential: bool = False, normalized_current: bool = False, correct_artifacts: bool = True,
              mask_nodata: bool = True, reclass_table=None, condition1=None, condition2=None,
              condition1_future=None, condition2_future=None, compare_to_future: str = "none",
              comparison1: str = "within", comparison2: str = "within", condition1_lower: float = 0.0,
              condition1_upper: float = 0.0, condition2_lower: float = 0.0, condition2_upper: float = 0.0,
              precision: str = "double", memory_limit: float | None = None, n_threads: int = 0,
              solver: str = "fp32-refine", preconditioner: str = "auto", edge_weights: str = "average",
              tol: float = 1e-12, device=None, return_stats: bool = False, checkpoint=None,
              chunk_windows: int | None = None):
    """Omnidirectional connectivity with Omniscape's moving-window circuits, solved on one GPU.

    Arguments, defaults and results are those of landschaft's ``ls.omniscape``
    (``omniscape.py:192-404``): every ``block_size`` x ``block_size`` block
    whose sources add up to more than 0 is a target; its window is the circle
    of ``radius + buffer`` around the block centre; the block's strength is
    injected into the sources within ``radius`` (the target block left out),
    the target cell is grounded, and the window's node currents are added to
    the cumulative map in a fixed order (bitwise reproducible).

    Added arguments: ``solver`` (``"fp32-refine"``: CG iterations in FP32 inside
    FP64 iterative refinement; ``"fp64"``: FP64 CG), ``preconditioner``
    (``"auto"``, ``"jacobi"``, ``"mg"``), ``edge_weights`` (``"average"``, as
    Omniscape; ``"series"``: resistor-series weights), ``tol`` (relative FP64
    residual of every window solve), ``device``, ``return_stats``, and streaming with resume: ``chunk_windows``
    solves the targets in consecutive ranges of that many windows (bitwise the same maps), ``checkpoint`` (an
    ``.npz`` path) saves the partial maps after every range and resumes from them.
    ``n_threads`` is accepted and has no effect; ``memory_limit`` bounds the
    device memory of one batch of window buffers.

    Returns an ``xarray.Dataset`` when xarray is importable, else a
    :class:`Dataset` with the same variables and ``attrs``.
    """
    import torch

    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}")
    dtype = np.float32 if precision == "single" else np.float64
    r, like = _grid(resistance, "resistance")
    if dtype is np.float32:
        r = r.astype(np.float32).astype(np.float64)
    if np.any(r <= 0):  # NaN (NoData) compares false
        raise ValueError("resistance (or conductance) values must be > 0")
    radius = _to_int(radius, "radius")
    buffer = _to_int(buffer, "buffer")
    block_size = _to_int(block_size, "block_size")
    if radius < 0 or buffer < 0 or block_size < 1:
        raise ValueError("radius and buffer must be >= 0 and block_size >= 1")
    if block_size % 2 == 0:
        warnings.warn("block_size is even, but must be odd. Using block_size + 1.", stacklevel=2)
        block_size += 1
    if source is None:
        s = source_from_resistance(r, r_cutoff=r_cutoff, resistance_is_conductance=resistance_is_conductance,
                                   reclass_table=reclass_table)
    else:
        s, _ = _grid(source, "source")
        if s.shape != r.shape:
            raise ValueError("the source raster must have the resistance's shape")
        if dtype is np.float32:
            s = s.astype(np.float32).astype(np.float64)
        s = np.where(np.isnan(s) | (s < source_threshold), 0.0, s)
    s = np.ascontiguousarray(s, dtype=np.float64)
    if reclass_table is not None:
        r = reclassify(r, reclass_table)
        if dtype is np.float32:
            r = r.astype(np.float32).astype(np.float64)
        if np.any(r <= 0):
            raise ValueError("the reclassified resistance must be > 0")
    r = np.ascontiguousarray(r)

    conditions = {}
    if condition2 is not None and condition1 is None:
        raise ValueError("condition2 needs condition1")
    if condition1 is not None:
        if compare_to_future not in COMPARE_TO_FUTURE:
            raise ValueError(f"compare_to_future must be one of {COMPARE_TO_FUTURE}")
        for k, cmp in ((1, comparison1), (2, comparison2)):
            if cmp not in COMPARISONS:
                raise ValueError(f"comparison{k} must be one of {COMPARISONS}")
        future1 = condition1_future if compare_to_future in ("1", "both") else None
        future2 = condition2_future if compare_to_future in ("2", "both") else None
        if compare_to_future in ("1", "both") and condition1_future is None:
            raise ValueError("compare_to_future needs condition1_future")
        if compare_to_future in ("2", "both") and condition2 is not None and condition2_future is None:
            raise ValueError("compare_to_future needs condition2_future")
        conditions = {
            "condition1": _condition(condition1, r.shape, "condition1", dtype),
            "condition1_future": _condition(future1, r.shape, "condition1_future", dtype),
            "condition2": _condition(condition2, r.shape, "condition2", dtype),
            "condition2_future": _condition(future2, r.shape, "condition2_future", dtype),
            "comparison1": comparison1, "comparison2": comparison2,
            "condition1_lower": float(condition1_lower), "condition1_upper": float(condition1_upper),
            "condition2_lower": float(condition2_lower), "condition2_upper": float(condition2_upper),
        }
    elif any(c is not None for c in (condition1_future, condition2_future)):
        raise ValueError("future conditions need condition1")

    compute_fp = bool(flow_potential or normalized_current)
    dev = _device(device)
    rt = torch.from_numpy(r).to(dev, non_blocking=False)
    stt = torch.from_numpy(s).to(dev)
    dcond = {}
    for k, v in conditions.items():
        dcond[k] = torch.from_numpy(v).to(dev) if isinstance(v, np.ndarray) else v
    params = make_params(radius, buffer, block_size, four_neighbors, resistance_is_conductance, correct_artifacts,
                         compute_fp, edge_weights, solver, preconditioner, tol, mask_nodata=mask_nodata,
                         memory_limit=memory_limit or 0.0, conditions=dcond or None)
    if chunk_windows or checkpoint is not None:
        out, stats = run_device_streamed(rt, stt, params, chunk_windows=int(chunk_windows or 100000),
                                         checkpoint=checkpoint, normalized=bool(normalized_current))
    else:
        out, stats = run_device(rt, stt, params, normalized=bool(normalized_current))
    cum = out["current"].cpu().numpy()
    data = {"cum_currmap": cum}
    if compute_fp:
        if normalized_current:
            data["normalized_cum_currmap"] = out["normalized"].cpu().numpy()
        if flow_potential:
            data["flow_potential"] = out["flow_potential"].cpu().numpy()
    if dtype is np.float32:
        data = {k: v.astype(np.float32) for k, v in data.items()}
    attrs = {"radius": radius, "block_size": block_size, "buffer": buffer, "n_targets": int(stats.n_targets),
             "four_neighbors": int(bool(four_neighbors)), "correct_artifacts": int(bool(correct_artifacts)),
             "precision": precision, "conditional": int(condition1 is not None), "threads": 1,
             "solver": solver, "cg_iterations_max": int(stats.iters_max),
             "cg_iterations_mean": float(stats.iters_total / max(stats.n_solved, 1)),
             "refinement_steps_max": int(stats.refine_max), "worst_relative_residual": float(stats.worst_residual)}
    ds = _dataset(data, attrs, like)
    if return_stats:
        return ds, stats.as_dict()
    return ds
