"""ctypes bindings of the two CPU oracles (test infrastructure only).

* ``liborc.so``: the C restatement in ``omni_oracle.c`` (the "port").
* ``_ref/libref_omni.so``: the reference's own ``omniscape.cpp``/``grid.cpp``
  compiled with the CellSystem of ``ref_shim.cpp`` (the "reference"); present
  only where it was built from the reference sources.

``omniscape`` below restates the reference's Python wrapper
(``src/landschaft/circuit/omniscape.py:192-404``: rounding, even block size,
default sources, thresholds, reclassification, conditions, normalised current,
NoData mask, single precision) around either library, returning a plain dict.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import warnings
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_PORT = HERE / "liborc.so"
_REF = HERE / "_ref" / "libref_omni.so"

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


_port = None
_ref = None


def port_lib():
    """The restatement's library, built with ``make`` when it is missing."""
    global _port
    if _port is None:
        if not _PORT.exists():
            subprocess.run(["make", "-C", str(HERE), "liborc.so"], check=True, capture_output=True)
        lib = C.CDLL(str(_PORT))
        lib.orc_omniscape.restype = C.c_int
        lib.orc_omniscape.argtypes = [_dp, _dp, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_int, C.c_double, C.c_double, _dp, _dp,
                                      C.c_int, C.c_double, C.c_double, C.c_int, C.c_int64, _dp, _dp, _i64p]
        lib.orc_correction.restype = C.c_int
        lib.orc_correction.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int64, _dp]
        lib.orc_advanced.restype = C.c_int
        lib.orc_advanced.argtypes = [_dp, _dp, _dp, C.c_int64, C.c_int64, C.c_int, C.c_int, _dp, _dp]
        lib.orc_count_targets.restype = C.c_int64
        lib.orc_count_targets.argtypes = [_dp, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int]
        lib.orc_omniscape_grad.restype = C.c_int
        lib.orc_omniscape_grad.argtypes = [_dp, _dp, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, _dp]
        _port = lib
    return _port


def ref_lib():
    """The reference-compiled library, or None where it was not built."""
    global _ref
    if _ref is None and _REF.exists():
        lib = C.CDLL(str(_REF))
        lib.ref_omniscape.restype = C.c_int
        lib.ref_omniscape.argtypes = [_dp, _dp, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, _dp, _dp, C.c_int, C.c_double, C.c_double, _dp, _dp, C.c_int,
                                      C.c_double, C.c_double, C.c_double, C.c_int, _dp, _dp, _i64p,
                                      C.POINTER(C.c_int), C.c_char_p, C.c_size_t]
        lib.ref_correction.restype = C.c_int
        lib.ref_correction.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int64, _dp, C.c_char_p,
                                       C.c_size_t]
        lib.ref_advanced.restype = C.c_int
        lib.ref_advanced.argtypes = [_dp, _dp, _dp, C.c_int64, C.c_int64, C.c_int, C.c_int, _dp, _dp, C.c_char_p,
                                     C.c_size_t]
        _ref = lib
    return _ref


REF_AVAILABLE = _REF.exists()

_ERRORS = {-1: "an Omniscape window is not positive definite", -2: "out of memory",
           -3: "a target block has no value of a condition (all NoData)",
           -4: "radius and buffer must be >= 0 and block_size odd"}


def _c64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _conditions(cond):
    """(present, future, equal, lower, upper) x 2 from the reference binding's dict (python.cpp:96-118)."""
    out = []
    for k in (1, 2):
        c = cond.get(f"condition{k}") if cond else None
        if c is None:
            out.append((None, None, 0, 0.0, 0.0))
            continue
        f = cond.get(f"condition{k}_future")
        out.append((_c64(c), _c64(f), int(cond[f"comparison{k}"] == "equal"), float(cond[f"condition{k}_lower"]),
                    float(cond[f"condition{k}_upper"])))
    return out


def core_omniscape(r, s, radius, buffer, block_size, four, ric, correct, fp, *, conditions=None, series=False,
                   threads=0, max_targets=-1, impl="port", memory_limit=0.0):
    """The native call (``circuit_omniscape``, python.cpp:90-137) on either oracle."""
    r = _c64(r)
    s = _c64(s)
    ny, nx = r.shape
    cur = np.zeros((ny, nx))
    fpo = np.zeros((ny, nx)) if fp else None
    nt = C.c_int64(0)
    (c1, c1f, c1e, c1l, c1u), (c2, c2f, c2e, c2l, c2u) = _conditions(conditions)
    if impl == "port":
        rc = port_lib().orc_omniscape(_ptr(r), _ptr(s), nx, ny, radius, buffer, block_size, int(four), int(ric),
                                      int(correct), int(fp), int(series), _ptr(c1), _ptr(c1f), c1e, c1l, c1u, _ptr(c2),
                                      _ptr(c2f), c2e, c2l, c2u, int(threads), int(max_targets), _ptr(cur), _ptr(fpo),
                                      C.byref(nt))
        if rc:
            raise (ValueError if rc == -4 else RuntimeError)(_ERRORS.get(rc, f"oracle error {rc}"))
        return {"current": cur, "flow_potential": fpo, "n_targets": nt.value, "threads": threads}
    if series:
        raise ValueError("the reference driver has no resistor-series option")
    lib = ref_lib()
    if lib is None:
        raise RuntimeError("the reference-compiled oracle was not built (oracle/_ref)")
    used = C.c_int(0)
    err = C.create_string_buffer(512)
    rc = lib.ref_omniscape(_ptr(r), _ptr(s), nx, ny, radius, buffer, block_size, int(four), int(ric), int(correct),
                           int(fp), _ptr(c1), _ptr(c1f), c1e, c1l, c1u, _ptr(c2), _ptr(c2f), c2e, c2l, c2u,
                           float(memory_limit), int(threads), _ptr(cur), _ptr(fpo), C.byref(nt), C.byref(used), err,
                           512)
    if rc:
        raise (ValueError if rc == 1 else RuntimeError)(err.value.decode())
    return {"current": cur, "flow_potential": fpo, "n_targets": nt.value, "threads": used.value}


def correction(radius, buffer, block_size, four, nx, ny, *, series=False):
    w = 2 * (radius + buffer) + 1
    out = np.zeros((w, w))
    rc = port_lib().orc_correction(radius, buffer, block_size, int(four), int(series), nx, ny, _ptr(out))
    if rc:
        raise RuntimeError(_ERRORS.get(rc, f"oracle error {rc}"))
    return out


def ref_correction(radius, buffer, block_size, four, nx, ny):
    lib = ref_lib()
    w = 2 * (radius + buffer) + 1
    out = np.zeros((w, w))
    err = C.create_string_buffer(512)
    if lib.ref_correction(radius, buffer, block_size, int(four), nx, ny, _ptr(out), err, 512):
        raise RuntimeError(err.value.decode())
    return out


def advanced(g, s, gr, four=False, series=False):
    """Single-raster solve (grid.cpp:73-210) on the port: (current, voltage)."""
    g, s, gr = _c64(g), _c64(s), _c64(gr)
    ny, nx = g.shape
    cur = np.zeros((ny, nx))
    volt = np.zeros((ny, nx))
    rc = port_lib().orc_advanced(_ptr(g), _ptr(s), _ptr(gr), nx, ny, int(four), int(series), _ptr(cur), _ptr(volt))
    if rc:
        raise RuntimeError(_ERRORS.get(rc, f"oracle error {rc}"))
    return cur, volt


def ref_advanced(g, s, gr, four=False, threads=0):
    lib = ref_lib()
    g, s, gr = _c64(g), _c64(s), _c64(gr)
    ny, nx = g.shape
    cur = np.zeros((ny, nx))
    volt = np.zeros((ny, nx))
    err = C.create_string_buffer(512)
    if lib.ref_advanced(_ptr(g), _ptr(s), _ptr(gr), nx, ny, int(four), int(threads), _ptr(cur), _ptr(volt), err, 512):
        raise RuntimeError(err.value.decode())
    return cur, volt


def count_targets(source, radius, buffer, block_size):
    s = _c64(source)
    ny, nx = s.shape
    return int(port_lib().orc_count_targets(_ptr(s), nx, ny, radius, buffer, block_size))


def omniscape_grad(r, s, weight, radius, buffer=0, block_size=1, four=False, ric=False, series=False, threads=0):
    """FP64 adjoint: (J, dJ/dresistance, dJ/dsource) for J = sum(weight * cum_current)."""
    r, s, weight = _c64(r), _c64(s), _c64(weight)
    ny, nx = r.shape
    gr = np.zeros((ny, nx))
    gs = np.zeros((ny, nx))
    J = C.c_double(0)
    rc = port_lib().orc_omniscape_grad(_ptr(r), _ptr(s), nx, ny, radius, buffer, block_size, int(four), int(ric),
                                       int(series), _ptr(weight), int(threads), _ptr(gr), _ptr(gs), C.byref(J))
    if rc:
        raise RuntimeError(_ERRORS.get(rc, f"oracle error {rc}"))
    return J.value, gr, gs


# --- the reference's Python wrapper, restated (omniscape.py:46-404) ---------------------------------------------

def _to_int(value, name):
    v = float(value)
    if not np.isfinite(v):
        raise ValueError(f"{name} must be finite")
    return int(round(v))


def _reclassify(r, table):
    t = np.array(table, dtype=np.float64).reshape(-1, 2)
    out = r.copy()
    for old, new in t:
        out[r == old] = new
    return out


def source_from_resistance(r, r_cutoff=np.inf, resistance_is_conductance=False, reclass_table=None):
    r = np.array(r, dtype=np.float64)
    if reclass_table is not None:
        r = _reclassify(r, reclass_table)
    with np.errstate(divide="ignore"):
        s = r if resistance_is_conductance else 1 / r
    return np.where(np.isnan(s) | (s < 1 / float(r_cutoff)), 0.0, s)


def omniscape(resistance, radius, *, source=None, block_size=1, buffer=0, source_threshold=0.0, r_cutoff=np.inf,
              resistance_is_conductance=False, four_neighbors=False, flow_potential=False, normalized_current=False,
              correct_artifacts=True, mask_nodata=True, reclass_table=None, condition1=None, condition2=None,
              condition1_future=None, condition2_future=None, compare_to_future="none", comparison1="within",
              comparison2="within", condition1_lower=0.0, condition1_upper=0.0, condition2_lower=0.0,
              condition2_upper=0.0, precision="double", impl="port", series=False, threads=0):
    """The reference's ``ls.omniscape`` around an oracle; returns a dict of maps plus ``attrs``."""
    dtype = np.float32 if precision == "single" else np.float64
    r = np.array(np.ma.filled(np.ma.asarray(resistance, dtype=np.float64), np.nan), dtype=np.float64)
    if dtype is np.float32:
        r = r.astype(np.float32).astype(np.float64)
    finite = r[~np.isnan(r)]
    if finite.size and finite.min() <= 0:
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
        s = source_from_resistance(r, r_cutoff, resistance_is_conductance, reclass_table)
    else:
        s = np.array(source, dtype=np.float64)
        if s.shape != r.shape:
            raise ValueError("the source raster must have the resistance's shape")
        if dtype is np.float32:
            s = s.astype(np.float32).astype(np.float64)
        s = np.where(np.isnan(s), 0.0, s)
        s = np.where(s < source_threshold, 0.0, s)
    if reclass_table is not None:
        r = _reclassify(r, reclass_table)
        if dtype is np.float32:
            r = r.astype(np.float32).astype(np.float64)
    conditions = None
    if condition1 is not None:
        def cnd(v):
            if v is None:
                return None
            v = np.array(v, dtype=np.float64)
            return v.astype(np.float32).astype(np.float64) if dtype is np.float32 else v
        conditions = {
            "condition1": cnd(condition1),
            "condition1_future": cnd(condition1_future if compare_to_future in ("1", "both") else None),
            "condition2": cnd(condition2),
            "condition2_future": cnd(condition2_future if compare_to_future in ("2", "both") else None),
            "comparison1": comparison1, "comparison2": comparison2,
            "condition1_lower": condition1_lower, "condition1_upper": condition1_upper,
            "condition2_lower": condition2_lower, "condition2_upper": condition2_upper}
    compute_fp = bool(flow_potential or normalized_current)
    out = core_omniscape(r, s, radius, buffer, block_size, four_neighbors, resistance_is_conductance,
                         correct_artifacts, compute_fp, conditions=conditions, series=series, threads=threads,
                         impl=impl)
    cum = out["current"]
    data = {"cum_currmap": cum}
    nodata = np.isnan(r)
    if compute_fp:
        fp = out["flow_potential"]
        if normalized_current:
            with np.errstate(divide="ignore", invalid="ignore"):
                norm = cum / fp
            norm[np.isnan(norm)] = 0.0
            data["normalized_cum_currmap"] = norm
        if flow_potential:
            data["flow_potential"] = fp
    if mask_nodata:
        for v in data.values():
            v[nodata] = np.nan
    if dtype is np.float32:
        data = {k: v.astype(np.float32) for k, v in data.items()}
    data["attrs"] = {"radius": radius, "block_size": block_size, "buffer": buffer, "n_targets": out["n_targets"]}
    return data


os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")
