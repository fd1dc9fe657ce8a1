"""The advanced mode of landschaft (``ls.circuit.advanced``) on the GPU, for one raster or a batch of them.

Mirrors ``src/landschaft/circuit/advanced.py:69-135`` (arguments, validation, messages and the
``AdvancedResult(current, voltage)`` result); the native call ``circuit_advanced``
(``src/cpp/circuit/python.cpp:65-80``, engine ``circuit::advanced`` in ``src/cpp/circuit/grid.cpp:73-210``) is
replaced by ``lsb_rasters`` of the C ABI, which solves a whole batch of independent rasters in one launch: one
persistent CTA per raster, every connected component with a source and a ground solved by CG (FP32 with FP64
refinement and a multigrid preconditioner, or plain FP64 with Jacobi).
"""

from __future__ import annotations

import ctypes as C
from typing import NamedTuple

import numpy as np

from . import _native as N
from .omni import SOLVERS, _device, _grid, _state


class AdvancedResult(NamedTuple):
    """``current``: max(inflow, outflow) at every node (0 where nothing was solved); ``voltage``: node voltages
    (0 in components without a source or a ground, NaN on cells without a node)."""

    current: object
    voltage: object


def _inputs(conductance, source, ground):
    """The reference's checks and NaN handling (advanced.py:125-134)."""
    g, _ = _grid(conductance, "conductance")
    s, _ = _grid(source, "source")
    gr, _ = _grid(ground, "ground")
    if s.shape != g.shape or gr.shape != g.shape:
        raise ValueError("conductance, source and ground must have the same shape")
    if np.any(g == np.inf):
        raise ValueError("conductances must be finite")
    if np.any(gr[np.isfinite(gr)] < 0):
        raise ValueError("ground conductances cannot be negative")
    s = np.where(np.isnan(s), 0.0, s)
    gr = np.where(np.isnan(gr), 0.0, gr)
    g = np.where(np.isnan(g), 0.0, g)
    return g, s, gr


def raster_params(four_neighbors=False, solver="fp32-refine", tol=1e-12, max_iter=20000,
                  memory_limit=0.0, smem_limit_kb=0) -> N.RasterParams:
    if solver not in SOLVERS:
        raise ValueError(f"solver must be one of {SOLVERS}")
    p = N.default_raster_params()
    p.four_neighbors = int(bool(four_neighbors))
    p.precision = N.PREC_FP64 if solver == "fp64" else N.PREC_FP32_REFINE
    p.tol = float(tol)
    p.max_iter = int(max_iter)
    p.memory_limit = float(memory_limit or 0.0)
    p.smem_limit_kb = int(smem_limit_kb)
    return p


def run_rasters(g, s, gr, shapes, params: N.RasterParams, *, want_stats=True):
    """One call of ``lsb_rasters`` on packed device tensors (float64, the rasters back to back).

    ``shapes`` lists each raster's (ny, nx).  Returns ``(current, voltage, stats)``: packed device tensors, and
    the call's statistics (None with ``want_stats=False``, which returns without waiting).
    """
    import torch
    lib = N.load()
    n = len(shapes)
    ny = (C.c_int32 * n)(*[int(a) for a, _ in shapes])
    nx = (C.c_int32 * n)(*[int(b) for _, b in shapes])
    cells = sum(int(a) * int(b) for a, b in shapes)
    for t in (g, s, gr):
        if t.dtype != torch.float64 or not t.is_cuda or t.device != g.device or t.numel() != cells:
            raise ValueError("conductance, source and ground must be packed float64 tensors on one CUDA device")
    g, s, gr = g.contiguous(), s.contiguous(), gr.contiguous()
    st = _state(g.device)
    with st.lock:
        nbytes = C.c_size_t(0)
        err = C.create_string_buffer(1024)
        rc = lib.lsb_rasters_workspace_size(n, nx, ny, C.byref(params), C.byref(nbytes))
        N.check(rc, C.create_string_buffer(b"invalid raster sizes or parameters"))
        ws = st.workspace(nbytes.value)
        cur = torch.empty(cells, dtype=torch.float64, device=g.device)
        volt = torch.empty_like(cur)
        stats = N.Stats() if want_stats else None
        caller = torch.cuda.current_stream(g.device)
        st.stream.wait_stream(caller)
        rc = lib.lsb_rasters(n, nx, ny, g.data_ptr(), s.data_ptr(), gr.data_ptr(), C.byref(params), cur.data_ptr(),
                             volt.data_ptr(), ws.data_ptr(), ws.numel(),
                             C.byref(stats) if stats is not None else None, err, len(err), st.stream.cuda_stream)
        caller.wait_stream(st.stream)
        N.check(rc, err)
    return cur, volt, stats


def advanced_batch(rasters, *, four_neighbors: bool = False, solver: str = "fp32-refine", tol: float = 1e-12,
                   device=None, return_stats: bool = False):
    """``advanced`` on many independent rasters in one launch: ``rasters`` is a sequence of
    (conductance, source, ground) triples (any shapes); returns a list of ``AdvancedResult`` (numpy)."""
    import torch
    dev = _device(device)
    prepared = [_inputs(*r) for r in rasters]
    if not prepared:
        return ([], None) if return_stats else []
    shapes = [p[0].shape for p in prepared]
    packed = [torch.from_numpy(np.concatenate([p[k].ravel() for p in prepared])).to(dev) for k in range(3)]
    cur, volt, stats = run_rasters(*packed, shapes, raster_params(four_neighbors, solver, tol))
    cur, volt = cur.cpu().numpy(), volt.cpu().numpy()
    out, o = [], 0
    for ny, nx in shapes:
        k = ny * nx
        out.append(AdvancedResult(cur[o:o + k].reshape(ny, nx), volt[o:o + k].reshape(ny, nx)))
        o += k
    return (out, stats.as_dict()) if return_stats else out


def advanced(conductance, source, ground, *, four_neighbors: bool = False, n_threads: int = 0,
             solver: str = "fp32-refine", tol: float = 1e-12, device=None) -> AdvancedResult:
    """Currents and voltages of a raster circuit with sources and grounds (drop-in for ``ls.circuit.advanced``).

    Every cell with a conductance > 0 is a node joined to its 8 neighbours (4 with ``four_neighbors``) by the
    average conductance of the two cells, over sqrt 2 on the diagonals.  ``source`` injects current into its
    cells; ``ground`` connects cells to ground with the given conductance (``inf``: a direct ground at 0 V); a
    cell that is both loses its source.  Every connected component with a source and a ground is solved, and a
    node's current is the larger of its inflow and outflow, leaving out branch currents under 1e-8 of the
    component's largest.  ``n_threads`` is accepted for compatibility (the solve runs on the GPU); ``solver`` and
    ``tol`` choose the GPU solve.
    """
    del n_threads
    return advanced_batch([(conductance, source, ground)], four_neighbors=four_neighbors, solver=solver, tol=tol,
                          device=device)[0]
