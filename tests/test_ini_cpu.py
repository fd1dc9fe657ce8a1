"""The INI front-end on CPU: parsing as Omniscape's parse_cfg, the ESRI ASCII grid reader and writer, errors that
need no solve."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import landschaft_b200 as lsb
from landschaft_b200 import ini

GOLD = Path(__file__).resolve().parent / "golden"


def test_parse_ini(tmp_path):
    # the reference's own case (tests/test_omniscape_ini.py:27-30)
    f = tmp_path / "a.ini"
    f.write_text("[Input files]\nresistance_file = r.tif \nradius=5\nweird = a = b\nno equals here\n[x]\n")
    assert lsb.parse_ini(f) == {"resistance_file": "r.tif", "radius": "5", "weird": "a = b"}


def test_ascii_grid_reads_decimals_as_float32_and_integers_exactly(tmp_path):
    v, nodata, prof = lsb.read_ascii_grid(GOLD / "omniscape_input" / "resistance.asc")
    assert v.shape == (30, 30) and nodata == -9999 and v.dtype == np.float32
    assert v[0, 0] == np.float32(0.29243631)
    f = tmp_path / "i.asc"
    f.write_text("ncols 3\nnrows 2\nxllcorner 0\nyllcorner 0\ncellsize 2\nNODATA_value -1\n1 2 3\n4 -1 16777217\n")
    v, nodata, prof = lsb.read_ascii_grid(f)
    assert v.dtype == np.int64 and v[1, 2] == 16777217 and prof["transform"] == (0.0, 0.0, 2.0, 2, 3)
    w, _ = ini._read(f, np.float64)
    assert np.isnan(w[1, 1]) and w[1, 2] == 16777217.0


def test_ascii_grid_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    a = rng.random((4, 5))
    a[1, 2] = np.nan
    prof = {"transform": (10.0, 20.0, 0.5, 4, 5), "crs": None}
    ini.write_ascii_grid(tmp_path / "o.asc", a, prof, np.float64)
    b, prof2 = ini._read(tmp_path / "o.asc", np.float64)
    np.testing.assert_array_equal(np.isnan(b), np.isnan(a))
    m = ~np.isnan(a)
    np.testing.assert_array_equal(b[m], a[m].astype(np.float32))  # decimals come back as the band's float32
    assert prof2["transform"] == prof["transform"]


def test_required_keys(tmp_path):
    f = tmp_path / "b.ini"
    f.write_text("radius = 3\nproject_name = p\n")
    with pytest.raises(ValueError, match="resistance_file"):
        lsb.omniscape_ini(f, write_outputs=False)
