"""Host-side checks that need no GPU: the C ABI library and the Python layer's validation."""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import landschaft_b200 as lsb
from landschaft_b200 import _native as N
from landschaft_b200 import synthetic
from landschaft_b200.omni import Dataset, _to_int

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "lsb_omniscape.h"


def header_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(lsb_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = N.load()
    declared = header_functions()
    assert set(declared) >= {"lsb_omniscape", "lsb_omniscape_workspace_size", "lsb_omniscape_correction"}
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(N.EXPORTS)


def test_struct_layouts_match_the_header(tmp_path):
    # sizes and field offsets of the ctypes mirrors against the header compiled by the C compiler
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    fields = {"lsb_omni_condition": N.Condition, "lsb_omni_params": N.Params, "lsb_omni_stats": N.Stats,
              "lsb_raster_params": N.RasterParams, "lsb_graph_params": N.GraphParams,
              "lsb_graph_stats": N.GraphStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "lsb_omniscape.h"', "int main(void) {"]
    for cname, py in fields.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    for cname, py in fields.items():
        assert int(out[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(out[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_defaults():
    p = N.default_params()
    assert (p.radius, p.buffer, p.block_size) == (0, 0, 1)
    assert p.correct_artifacts == 1 and p.precision == N.PREC_FP32_REFINE and p.preconditioner == N.PC_AUTO
    assert p.tol == 1e-12 and p.use_graph == 1
    assert N.load().lsb_version().startswith(b"landschaft_b200")


def test_to_int_rounds_half_to_even():
    assert _to_int(2.5, "r") == 2 and _to_int(3.5, "r") == 4 and _to_int("7", "r") == 7
    with pytest.raises(ValueError, match="finite"):
        _to_int(float("inf"), "radius")


def test_bad_inputs_raise_before_the_device():
    r = np.exp(np.random.default_rng(8).normal(0.5, 1.0, (20, 25)))
    with pytest.raises(ValueError, match="> 0"):
        lsb.omniscape(np.where(r > 2, 0, r), 3)
    with pytest.raises(ValueError, match="shape"):
        lsb.omniscape(r, 3, source=np.ones((3, 3)))
    with pytest.raises(ValueError, match="precision"):
        lsb.omniscape(r, 3, precision="half")
    with pytest.raises(ValueError, match=">= 0"):
        lsb.omniscape(r, -1)
    with pytest.raises(ValueError, match="condition2 needs condition1"):
        lsb.omniscape(r, 3, condition2=r)
    with pytest.raises(ValueError, match="comparison1"):
        lsb.omniscape(r, 3, condition1=r, comparison1="near")
    with pytest.raises(ValueError, match="future conditions need condition1"):
        lsb.omniscape(r, 3, condition1_future=r)
    with pytest.raises(ValueError, match="2-D"):
        lsb.omniscape(np.ones(5), 3)


def test_no_cpu_fallback():
    # the product path raises without a CUDA device instead of computing on the CPU
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    r = np.ones((10, 10))
    with pytest.raises(RuntimeError, match="CUDA"):
        lsb.omniscape(r, 2)
    with pytest.warns(UserWarning, match="block_size is even"):
        with pytest.raises(RuntimeError, match="CUDA"):
            lsb.omniscape(r, 2, block_size=2)


def test_source_from_resistance_and_reclass(tmp_path):
    rng = np.random.default_rng(5)
    r = np.exp(rng.normal(0.5, 1.0, (12, 14)))
    r[rng.random(r.shape) < 0.1] = np.nan
    s = lsb.source_from_resistance(r, r_cutoff=2.0)
    np.testing.assert_array_equal(s, np.where(np.isnan(r) | (1 / r < 0.5), 0, 1 / r))
    np.testing.assert_array_equal(lsb.source_from_resistance(1 / r, resistance_is_conductance=True),
                                  np.where(np.isnan(r), 0, 1 / r))
    table = np.array([[1, 10], [2, 50], [3, np.nan]])
    np.testing.assert_array_equal(lsb.reclassify(np.array([[1.0, 2.0], [3.0, 4.0]]), table),
                                  [[10.0, 50.0], [np.nan, 4.0]])
    path = tmp_path / "reclass.txt"
    path.write_text("1 10\n2 50\n3 missing\n")
    np.testing.assert_array_equal(lsb.read_reclass_table(path), table)
    np.testing.assert_array_equal(lsb.reclassify(np.array([[1.0, 3.0]]), {1: 5, 3: None}), [[5.0, np.nan]])


def test_dataset_shape():
    ds = Dataset({"cum_currmap": np.zeros((2, 3)), "flow_potential": np.ones((2, 3))}, {"n_targets": 4})
    assert ds.data_vars == ["cum_currmap", "flow_potential"]
    assert "cum_currmap" in ds and ds.attrs["n_targets"] == 4
    assert ds.cum_currmap.values.shape == (2, 3) and ds["flow_potential"].values.sum() == 6


def test_active_blocks_and_window_cells_match_the_oracle():
    import oracle
    from landschaft_b200 import omni
    rng = np.random.default_rng(1)
    s = rng.random((37, 41))
    s[s < 0.7] = 0
    for bs in (1, 3, 5, 7):
        assert omni.active_blocks(s, bs).sum() == oracle.count_targets(s, 4, 0, bs)
    assert omni.window_cells((5, 6), {"radius": 1}) == sum(
        (min(y + 1, 4) - max(y - 1, 0) + 1) * (min(x + 1, 5) - max(x - 1, 0) + 1) for y in range(5) for x in range(6))


def test_synthetic_workloads():
    r, s, kw = synthetic.omni_128()
    assert r.shape == (128, 128) and r.min() >= 1 and r.max() <= 100
    np.testing.assert_array_equal(s, 1 / r)
    g = synthetic.gaussian_field(64, -3.0, 0)
    assert g.min() == 0 and g.max() == 1
    m = synthetic.nodata_clusters((100, 100), 0.01, 1)
    assert 0.005 < m.mean() < 0.02
    p = synthetic.nodata_polygons((300, 300), 0.05, 2)
    assert 0.05 <= p.mean() < 0.08
    # deterministic
    np.testing.assert_array_equal(synthetic.omni_grf(64, 3)[0], synthetic.omni_grf(64, 3)[0])


def test_tuning_table_set_get_clear_and_file(tmp_path):
    # the table is host state of the library: no device needed
    lib = N.load()
    lsb.clear_tuning()
    pc, nt = C.c_int32(-1), C.c_int32(-1)
    assert lib.lsb_tune_get(65, 0, 0, N.PREC_FP32_REFINE, C.byref(pc), C.byref(nt)) == 0
    assert lib.lsb_tune_set(65, 0, 0, N.PREC_FP32_REFINE, 3, 256) != 0  # no such preconditioner
    assert lib.lsb_tune_set(65, 0, 0, N.PREC_FP32_REFINE, 1, 384) != 0  # no such block size
    entry = {"window": 65, "four_neighbors": False, "edge_weights": "average", "solver": "fp32-refine",
             "preconditioner": "jacobi", "threads_per_window": 256}
    from landschaft_b200 import tune
    tune._install(entry)
    assert lib.lsb_tune_get(65, 0, 0, N.PREC_FP32_REFINE, C.byref(pc), C.byref(nt)) == 1
    assert (pc.value, nt.value) == (1, 256)
    assert lib.lsb_tune_get(65, 1, 0, N.PREC_FP32_REFINE, C.byref(pc), C.byref(nt)) == 0  # other neighbourhood
    path = tmp_path / "tuning.json"
    lsb.save_tuning(path)
    lsb.clear_tuning()
    assert lib.lsb_tune_get(65, 0, 0, N.PREC_FP32_REFINE, C.byref(pc), C.byref(nt)) == 0
    assert lsb.load_tuning(path) == 1
    assert lib.lsb_tune_get(65, 0, 0, N.PREC_FP32_REFINE, C.byref(pc), C.byref(nt)) == 1
    assert lsb.tuning_table()[0]["preconditioner"] == "jacobi"
    lsb.clear_tuning()
