"""Omniscape INI files on the GPU: the 11 Omniscape.jl runs the reference pins (tests/test_omniscape_ini.py:
124-145) against their CHOLMOD outputs (tests/golden/omniscape_ini.npz), with the same warnings and errors; the
outputs written to the project folder."""

from __future__ import annotations

import contextlib
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
INI = GOLD / "omniscape_ini"
OUTPUTS = ("cum_currmap", "flow_potential", "normalized_cum_currmap", "classified_resistance")
WARNS = ("config", "config3", "config5", "config_32bit")  # even block size, unknown keys, reclass table unused


@pytest.fixture(scope="module")
def lsb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import landschaft_b200
    return landschaft_b200


def _cases():
    z = np.load(GOLD / "omniscape_ini.npz")
    return sorted({k.split("/")[0] for k in z.files})


@pytest.mark.parametrize("name", _cases())
def test_matches_omniscape_ini(lsb, name):
    z = np.load(GOLD / "omniscape_ini.npz")
    ctx = pytest.warns(UserWarning) if name in WARNS else contextlib.nullcontext()
    with ctx:
        ds = lsb.omniscape_ini(INI / f"{name}.ini", write_outputs=False)
    single = name == "config_32bit"
    checked = 0
    for out in OUTPUTS:
        key = f"{name}/cholmod/{out}"
        if key not in z.files:
            continue
        ours = np.asarray(ds[out].values, dtype=float)
        chol = z[key]
        np.testing.assert_array_equal(np.isnan(ours), np.isnan(chol))
        np.testing.assert_array_equal(ours == 0, chol == 0)
        top = np.nanmax(np.abs(chol))
        if single:
            # Omniscape computes in float32, this build in double and rounds the result
            np.testing.assert_allclose(ours, chol, rtol=1e-3, atol=1e-3 * top)
        else:
            np.testing.assert_allclose(ours, chol, rtol=1e-9, atol=1e-13 * top)
        checked += 1
    assert checked


def test_resistance_of_zero_raises(lsb):
    # Omniscape's test configuration 7 has a resistance of 0
    with pytest.raises(ValueError, match="> 0"):
        lsb.omniscape_ini(INI / "config7.ini", write_outputs=False)


def test_writes_the_outputs(lsb, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    ds = lsb.omniscape_ini(INI / "config_reclass.ini")  # write_as_tif = false: ASCII grids
    out = Path(ds.attrs["project_dir"])
    assert sorted(p.name for p in out.iterdir()) == ["classified_resistance.asc", "config.ini", "cum_currmap.asc"]
    v, nodata, _ = lsb.read_ascii_grid(out / "cum_currmap.asc")
    want = np.asarray(ds["cum_currmap"].values, dtype=float)
    m = ~np.isnan(want)
    assert nodata == -9999 and np.all(v[~m] == -9999)
    np.testing.assert_array_equal(v[m], want[m].astype(np.float32))  # read back as the band's float32
    with pytest.warns(UserWarning, match="already exists"):
        ds2 = lsb.omniscape_ini(INI / "config_reclass.ini")
    assert ds2.attrs["project_dir"].endswith("_1")
