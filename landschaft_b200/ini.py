"""Omniscape's INI files on the GPU: the drop-in for ``ls.circuit.omniscape_ini`` (``run_omniscape(path)``).

Mirrors ``src/landschaft/circuit/ini.py`` of landschaft: the same parsing (``parse_ini``), required keys, defaults,
warnings and errors, and the same mapping of the options onto :func:`landschaft_b200.omniscape`; the windows are
solved on the GPU.  Rasters are read and written as ESRI ASCII grids by this module (the reference goes through
rasterio, absent here; GeoTIFF inputs and outputs use rasterio when it is importable).  An ASCII grid whose values
have a decimal point or an exponent is read as 32-bit floats, as GDAL's AAIGrid driver (and so the reference and
Omniscape.jl) reads it; one with integers only, exactly.
"""

from __future__ import annotations

import os
import re
import warnings
from pathlib import Path

import numpy as np

from .omni import omniscape, read_reclass_table, reclassify

TRUELIST = ("true", "True", "TRUE")
REQUIRED = ("resistance_file", "radius", "project_name")
SUPPORTED = (
    "resistance_file", "resistance_is_conductance", "source_file", "project_name", "parallelize",
    "parallel_batch_size", "block_size", "radius", "buffer", "source_threshold", "source_from_resistance",
    "r_cutoff", "precision", "connect_four_neighbors_only", "solver", "calc_flow_potential",
    "calc_normalized_current", "correct_artifacts", "write_raw_currmap", "write_as_tif", "mask_nodata",
    "suppress_cs_messages", "conditional", "n_conditions", "compare_to_future", "condition1_file",
    "condition2_file", "condition1_future_file", "condition2_future_file", "comparison1", "comparison2",
    "condition1_lower", "condition2_lower", "condition1_upper", "condition2_upper", "reclassify_resistance",
    "reclass_table", "write_reclassified_resistance", "allow_different_projections",
)
DEFAULTS = {
    "resistance_file": "", "resistance_is_conductance": "false", "source_file": "",
    "parallelize": "true", "parallel_batch_size": "10", "block_size": "1", "buffer": "0",
    "source_threshold": "0", "source_from_resistance": "false", "r_cutoff": "Inf", "precision": "double",
    "connect_four_neighbors_only": "false", "solver": "cg+amg", "calc_flow_potential": "false",
    "calc_normalized_current": "false", "correct_artifacts": "true", "write_raw_currmap": "true",
    "write_as_tif": "true", "mask_nodata": "true", "suppress_cs_messages": "true", "conditional": "false",
    "n_conditions": "1", "compare_to_future": "none", "condition1_file": "", "condition2_file": "",
    "condition1_future_file": "", "condition2_future_file": "", "comparison1": "within", "comparison2": "within",
    "condition1_lower": "0", "condition2_lower": "0", "condition1_upper": "0", "condition2_upper": "0",
    "reclassify_resistance": "false", "reclass_table": "", "write_reclassified_resistance": "false",
    "allow_different_projections": "false",
}


def parse_ini(path) -> dict:
    """Omniscape's ``parse_cfg``: lines starting with ``[`` are skipped; every other line with an ``=`` is split at
    its first ``=`` (key right-stripped, value stripped)."""
    cfg = {}
    with open(path, encoding="utf-8") as f:
        for line in f:
            if line.startswith("["):
                continue
            key, sep, value = line.partition("=")
            if sep:
                cfg[key.rstrip()] = value.strip()
    return cfg


def _float(value: str) -> float:
    # Julia's parse(Float64, ...) also takes Inf and NaN
    return float(value.replace("Inf", "inf"))


# ---------------------------------------------------------------------------------------------------------------
# ESRI ASCII grids
# ---------------------------------------------------------------------------------------------------------------

_HEADER_KEYS = ("ncols", "nrows", "xllcorner", "yllcorner", "xllcenter", "yllcenter", "cellsize", "nodata_value",
                "dx", "dy")


def read_ascii_grid(path):
    """(values float64 with the band's rounding, nodata value or None, profile) of an ESRI ASCII grid."""
    text = Path(path).read_text()
    tokens = text.split()
    head, k = {}, 0
    while k + 1 < len(tokens) and tokens[k].lower() in _HEADER_KEYS:
        head[tokens[k].lower()] = tokens[k + 1]
        k += 2
    ncols, nrows = int(head["ncols"]), int(head["nrows"])
    body = tokens[k:k + ncols * nrows]
    if len(body) != ncols * nrows:
        raise ValueError(f"{path}: expected {nrows} x {ncols} values")
    floating = any(re.search(r"[.eE]", t) for t in body)
    band = np.float32 if floating else np.int64
    a = np.array([float(t) for t in body], dtype=np.float64).astype(band).reshape(nrows, ncols)
    nodata = float(head["nodata_value"]) if "nodata_value" in head else None
    cell = float(head.get("cellsize", head.get("dx", "1")))
    x0 = float(head["xllcorner"]) if "xllcorner" in head else float(head.get("xllcenter", "0")) - cell / 2
    y0 = float(head["yllcorner"]) if "yllcorner" in head else float(head.get("yllcenter", "0")) - cell / 2
    prj = Path(path).with_suffix(".prj")
    profile = {"transform": (x0, y0, cell, nrows, ncols), "crs": prj.read_text().strip() if prj.exists() else None,
               "band": band}
    return a, nodata, profile


def write_ascii_grid(path, values, profile, dtype, nodata=-9999):
    x0, y0, cell, _, _ = profile["transform"]
    ny, nx = values.shape
    out = np.where(np.isnan(values), nodata, values).astype(dtype)
    lines = [f"ncols {nx}", f"nrows {ny}", f"xllcorner {x0!r}", f"yllcorner {y0!r}", f"cellsize {cell!r}",
             f"NODATA_value {nodata}"]
    fmt = "%.9g" if out.dtype == np.float32 else "%.17g"
    lines += [" ".join(fmt % v for v in row) for row in out]
    Path(path).write_text("\n".join(lines) + "\n")
    if profile.get("crs"):
        Path(path).with_suffix(".prj").write_text(profile["crs"])


def _resolve(name: str, base: Path) -> Path:
    # Omniscape reads paths from the working directory; failing that, next to the INI file
    p = Path(name)
    if p.is_absolute() or p.exists():
        return p
    q = base / p
    return q if q.exists() else p


def _read(path: Path, dtype):
    """A raster as Omniscape's ``read_raster``: band 1, nodata (in the band's type) and NaN missing."""
    if not path.exists():
        raise FileNotFoundError(f'the file "{path}" does not exist')
    if path.suffix.lower() in (".asc", ".txt"):
        a, nodata, profile = read_ascii_grid(path)
    else:
        try:
            import rasterio
        except ImportError as e:
            raise ValueError(f"{path}: only ESRI ASCII grids can be read without rasterio") from e
        with rasterio.open(path) as src:
            a = src.read(1)
            nodata = src.nodata
            t = src.transform
            profile = {"transform": (t.c, t.f - src.height * t.a, t.a, src.height, src.width),
                       "crs": str(src.crs) if src.crs else None, "band": a.dtype}
    band = profile["band"]
    v = a.astype(dtype).astype(np.float64)
    if nodata is not None:
        v[v == np.array(nodata).astype(band).astype(dtype).astype(np.float64)] = np.nan
    return v, profile


def _aligned(ref, other, name1, name2, allow_projections: bool) -> None:
    (a, pa), (b, pb) = ref, other
    if pa["crs"] != pb["crs"] or pa["transform"] != pb["transform"]:
        if not allow_projections:
            warnings.warn(f"{name1} and {name2} have different projections. This could mean they are not properly "
                          "aligned. Attempting to proceed anyway.", stacklevel=3)
    if a.shape != b.shape:
        raise ValueError(f"{name1} and {name2} are different sizes.")


def _project_dir(name: str) -> Path:
    base = Path(name)
    if not base.is_dir():
        base.mkdir(parents=True, exist_ok=True)
        return base
    k = 1
    while Path(f"{name}_{k}").is_dir():
        k += 1
    out = Path(f"{name}_{k}")
    warnings.warn(f"Your specified project directory, {name}, already exists. Writing outputs to {out}.",
                  stacklevel=3)
    out.mkdir(parents=True)
    return out


def _write(path: Path, values, profile, tif: bool, dtype) -> None:
    if tif:
        try:
            import rasterio
            from rasterio.transform import from_origin
        except ImportError:
            warnings.warn("GeoTIFF output needs rasterio; writing an ESRI ASCII grid instead", stacklevel=3)
        else:
            x0, y0, cell, ny, nx = profile["transform"]
            out = np.where(np.isnan(values), -9999, values).astype(dtype)
            with rasterio.open(path.with_suffix(".tif"), "w", driver="GTiff", height=ny, width=nx, count=1,
                               dtype=out.dtype, nodata=-9999, crs=profile["crs"],
                               transform=from_origin(x0, y0 + ny * cell, cell, cell)) as dst:
                dst.write(out, 1)
            return
    write_ascii_grid(path.with_suffix(".asc"), values, profile, dtype)


def omniscape_ini(path, *, write_outputs: bool = True, n_threads: int = 0, solver: str = "fp32-refine",
                  tol: float = 1e-12, device=None):
    """Run an Omniscape INI file, as ``run_omniscape(path)`` does (drop-in for ``ls.circuit.omniscape_ini``).

    Every option of Omniscape 0.7 is read with its defaults (``radius``, ``resistance_file`` and
    ``project_name`` are required); file paths are taken from the working directory, or else next to the INI
    file.  With ``write_outputs`` the outputs go to ``project_name`` (``_1``, ``_2``... when it exists):
    ``config.ini``, ``cum_currmap``, ``flow_potential``, ``normalized_cum_currmap`` and
    ``classified_resistance``, NoData -9999.  The INI's ``solver``, ``parallelize``, ``parallel_batch_size`` and
    ``suppress_cs_messages`` have no effect; ``solver`` and ``tol`` of this call choose the GPU solve.
    """
    del n_threads
    path = Path(path)
    base = path.resolve().parent
    user = parse_ini(path)
    missing = [k for k in REQUIRED if k not in user]
    if missing:
        raise ValueError("The following arguments are missing from your .ini with no defaults: " + " ".join(missing))
    unknown = [k for k in user if k not in SUPPORTED and k != ""]
    if unknown:
        warnings.warn("The following unsupported arguments were provided and will be ignored: " + " ".join(unknown),
                      stacklevel=2)
    cfg = {**DEFAULTS, **user}
    flag = {k: cfg[k] in TRUELIST for k in cfg}
    precision = "single" if cfg["precision"] in ("single", "Single", "SINGLE") else "double"
    dtype = np.float32 if precision == "single" else np.float64
    allow = flag["allow_different_projections"]

    res = _read(_resolve(cfg["resistance_file"], base), dtype)
    resistance = res[0]
    reclass = None
    if flag["reclassify_resistance"]:
        reclass = read_reclass_table(_resolve(cfg["reclass_table"], base))
    elif cfg["reclass_table"] != "":
        warnings.warn("You provided a reclass_table, but did not set reclassify_resistance to true. Resistance will "
                      "not be reclassified.", stacklevel=2)

    source = None
    if not flag["source_from_resistance"]:
        if cfg["source_file"] == "":
            raise ValueError("You did not provide a source raster file path. Set source_from_resistance to true in "
                             "your config if you want to generate source strength from the resistance layer.")
        src = _read(_resolve(cfg["source_file"], base), dtype)
        _aligned(res, src, "resistance_file", "source_file", allow)
        source = src[0]

    conds = {}
    if flag["conditional"]:
        compare = cfg["compare_to_future"].lower()
        n_cond = int(round(_float(cfg["n_conditions"])))

        def cond(key):
            c = _read(_resolve(cfg[key], base), dtype)
            _aligned(res, c, "resistance_file", key, allow)
            return c[0]

        conds["condition1"] = cond("condition1_file")
        if compare in ("1", "both"):
            conds["condition1_future"] = cond("condition1_future_file")
        if n_cond == 2:
            conds["condition2"] = cond("condition2_file")
            if compare in ("2", "both"):
                conds["condition2_future"] = cond("condition2_future_file")
        elif n_cond != 1:
            raise ValueError(f"n_conditions must be one of ['1', '2']. Got {cfg['n_conditions']}.")
        conds.update(compare_to_future=compare, comparison1=cfg["comparison1"], comparison2=cfg["comparison2"],
                     condition1_lower=_float(cfg["condition1_lower"]), condition1_upper=_float(cfg["condition1_upper"]),
                     condition2_lower=_float(cfg["condition2_lower"]), condition2_upper=_float(cfg["condition2_upper"]))
    elif cfg["condition1_file"] != "" or cfg["condition2_file"] != "":
        warnings.warn("conditional is set to false in your INI but you provided file paths to condition files.",
                      stacklevel=2)

    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)  # block_size: warned below, once
        ds = omniscape(
            resistance, _float(cfg["radius"]), source=source, block_size=_float(cfg["block_size"]),
            buffer=_float(cfg["buffer"]), source_threshold=_float(cfg["source_threshold"]),
            r_cutoff=_float(cfg["r_cutoff"]), resistance_is_conductance=flag["resistance_is_conductance"],
            four_neighbors=flag["connect_four_neighbors_only"], flow_potential=flag["calc_flow_potential"],
            normalized_current=flag["calc_normalized_current"], correct_artifacts=flag["correct_artifacts"],
            mask_nodata=flag["mask_nodata"], reclass_table=reclass, precision=precision, solver=solver, tol=tol,
            device=device, **conds)
    if int(round(_float(cfg["block_size"]))) % 2 == 0:
        warnings.warn("block_size is even, but must be odd. Using block_size + 1.", stacklevel=2)
    if reclass is not None:
        ds["classified_resistance"] = (("y", "x"), reclassify(resistance, reclass).astype(dtype))

    if write_outputs:
        out = _project_dir(cfg["project_name"])
        with open(out / "config.ini", "a", encoding="utf-8") as f:
            for k, v in user.items():
                if k:
                    f.write(f"{k} = {v}\n")
        tif = flag["write_as_tif"]
        profile = res[1]
        if reclass is not None and flag["write_reclassified_resistance"]:
            _write(out / "classified_resistance", np.asarray(ds["classified_resistance"].values), profile, tif, dtype)
        if flag["write_raw_currmap"]:
            _write(out / "cum_currmap", np.asarray(ds["cum_currmap"].values), profile, tif, dtype)
        if flag["calc_flow_potential"]:
            _write(out / "flow_potential", np.asarray(ds["flow_potential"].values), profile, tif, dtype)
        if flag["calc_normalized_current"]:
            _write(out / "normalized_cum_currmap", np.asarray(ds["normalized_cum_currmap"].values), profile, tif,
                   dtype)
        ds.attrs["project_dir"] = os.fspath(out)
    return ds
