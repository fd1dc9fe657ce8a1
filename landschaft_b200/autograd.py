"""Gradients of the cumulative current with respect to the resistance and source rasters.

The reference has no adjoint; this is an addition of the GPU build.  ``lsb_omniscape_grad`` (C ABI) computes,
for J = sum(weight * cumulative current), dJ/d(resistance) and dJ/d(source): every window's forward potentials
are recomputed (not stored), the derivative of its node currents with respect to the potentials is the
right-hand side of one more solve with the same symmetric operator (the adjoint), and the chain rule runs through
the edge weights, g = 1/r and the scaling of the sources to the block's amps.

``omniscape_current`` wraps forward and backward in a ``torch.autograd.Function``: its backward calls the adjoint
with the incoming gradient map as ``weight`` (the vector-Jacobian product).
"""

from __future__ import annotations

import ctypes as C

from . import _native as N
from .omni import _state, make_params, run_device


def grad_device(r, s, weight, params: N.Params, *, want_source=True):
    """dJ/dr, dJ/ds and J for J = sum(weight * cumulative current); device float64 tensors in and out.

    ``params`` must have no block-artifact correction (block size 1, or correct_artifacts off) and no
    conditions.  Returns ``(J, grad_r, grad_s, stats)``; grad_s is None when ``want_source`` is false.
    """
    import torch
    lib = N.load()
    for t in (r, s, weight):
        if t.dtype != torch.float64 or not t.is_cuda or t.device != r.device or t.shape != r.shape:
            raise ValueError("resistance, source and weight must be float64 tensors of one shape on one CUDA device")
    r, s, weight = r.contiguous(), s.contiguous(), weight.contiguous()
    ny, nx = r.shape
    st = _state(r.device)
    with st.lock:
        nbytes = C.c_size_t(0)
        err = C.create_string_buffer(1024)
        rc = lib.lsb_omniscape_grad_workspace_size(nx, ny, C.byref(params), C.byref(nbytes))
        N.check(rc, C.create_string_buffer(b"invalid parameters"))
        ws = st.workspace(nbytes.value)
        gr = torch.empty_like(r)
        gs = torch.empty_like(r) if want_source else None
        J = torch.empty(1, dtype=torch.float64, device=r.device)
        stats = N.Stats()
        cur = torch.cuda.current_stream(r.device)
        st.stream.wait_stream(cur)
        rc = lib.lsb_omniscape_grad(r.data_ptr(), s.data_ptr(), weight.data_ptr(), nx, ny, C.byref(params),
                                    gr.data_ptr(), gs.data_ptr() if gs is not None else None, J.data_ptr(),
                                    ws.data_ptr(), ws.numel(), C.byref(stats), err, len(err), st.stream.cuda_stream)
        cur.wait_stream(st.stream)
        N.check(rc, err)
    return J, gr, gs, stats


def _function():
    import torch

    class OmniscapeCurrent(torch.autograd.Function):
        """Cumulative current as a differentiable function of (resistance, source)."""

        @staticmethod
        def forward(ctx, resistance, source, kwargs):
            p = make_params(**kwargs)
            out, _ = run_device(resistance, source, p)
            ctx.save_for_backward(resistance, source)
            ctx.kwargs = kwargs
            return out["current"]

        @staticmethod
        def backward(ctx, grad_current):
            resistance, source = ctx.saved_tensors
            p = make_params(**ctx.kwargs)
            w = grad_current.contiguous().to(torch.float64)
            w = torch.nan_to_num(w, nan=0.0)
            _, gr, gs, _ = grad_device(resistance, source, w, p, want_source=ctx.needs_input_grad[1])
            return gr if ctx.needs_input_grad[0] else None, gs, None

    return OmniscapeCurrent


_FN = None


def omniscape_current(resistance, source, radius, *, buffer=0, block_size=1, four_neighbors=False,
                      resistance_is_conductance=False, edge_weights="average", solver="fp32-refine",
                      preconditioner="auto", tol=1e-12):
    """Differentiable cumulative current (device float64 tensors; NaN resistance = NoData).

    Sources are taken as given (apply thresholds and NaN -> 0 before, as ``omniscape`` does); block_size > 1 runs
    without the block-artifact correction.  ``torch.autograd`` gives d/d(resistance) and d/d(source).
    """
    global _FN
    if _FN is None:
        _FN = _function()
    kwargs = dict(radius=int(radius), buffer=int(buffer), block_size=int(block_size),
                  four_neighbors=bool(four_neighbors), resistance_is_conductance=bool(resistance_is_conductance),
                  correct_artifacts=False, flow_potential=False, edge_weights=edge_weights, solver=solver,
                  preconditioner=preconditioner, tol=tol, use_graph=False)
    return _FN.apply(resistance, source, kwargs)
