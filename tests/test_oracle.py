"""The CPU oracle against the reference's golden vectors and known answers (no GPU).

Pins ``oracle/omni_oracle.c`` (the C restatement) and, where it was built,
``oracle/_ref`` (the reference's own driver) to:

* the 8 Omniscape.jl 0.7 + CHOLMOD cases of the reference's
  ``tests/data/reference/circuit/omniscape.npz`` (tests/test_omniscape.py:131-161
  of the reference: identical NaN and zero patterns, rtol 1e-9, atol 1e-13 max);
* the 6 Circuitscape advanced-mode CHOLMOD cases (tests/test_circuit.py:135-148);
* the known answers of the reference's docstrings and tests.
"""

from __future__ import annotations

import json
import warnings
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLD = Path(__file__).parent / "golden"
OUTPUTS = ("cum_currmap", "flow_potential", "normalized_cum_currmap")
OPTION_NAMES = {"connect_four_neighbors_only": "four_neighbors", "calc_flow_potential": "flow_potential",
                "calc_normalized_current": "normalized_current"}


def golden_cases():
    z = np.load(GOLD / "omniscape_golden.npz")
    return sorted({k.split("/")[0] for k in z.files})


def golden_kwargs(z, name):
    options = json.loads(str(z[f"{name}/options"]))
    kw = {OPTION_NAMES.get(k, k): v for k, v in options.items() if k != "source_from_resistance"}
    source = None if options.get("source_from_resistance") else z[f"{name}/source"]
    return kw, source


def check_golden(out, z, name, rtol=1e-9, atol_rel=1e-13):
    checked = 0
    for o in OUTPUTS:
        key = f"{name}/cholmod/{o}"
        if key not in z.files:
            assert o not in out
            continue
        ours, chol = np.asarray(out[o]), z[key]
        np.testing.assert_array_equal(np.isnan(ours), np.isnan(chol))
        np.testing.assert_array_equal(ours == 0, chol == 0)
        np.testing.assert_allclose(ours, chol, rtol=rtol, atol=atol_rel * np.nanmax(chol))
        checked += 1
    assert checked


def _map(seed=1, shape=(40, 50)):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.normal(0.5, 1.0, shape))
    r[rng.random(shape) < 0.05] = np.nan
    return r


@pytest.mark.parametrize("name", golden_cases())
def test_port_matches_omniscape_golden(name):
    z = np.load(GOLD / "omniscape_golden.npz")
    kw, source = golden_kwargs(z, name)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        out = oracle.omniscape(z[f"{name}/resistance"], source=source, **kw)
    check_golden(out, z, name)


@pytest.mark.skipif(not oracle.REF_AVAILABLE, reason="the reference-compiled oracle was not built here")
@pytest.mark.parametrize("name", golden_cases())
def test_reference_build_matches_omniscape_golden(name):
    z = np.load(GOLD / "omniscape_golden.npz")
    kw, source = golden_kwargs(z, name)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        out = oracle.omniscape(z[f"{name}/resistance"], source=source, impl="ref", **kw)
    check_golden(out, z, name)


def _advanced_cases():
    a = np.load(GOLD / "advanced_golden.npz")
    return sorted({k.split("/")[0] for k in a.files})


@pytest.mark.parametrize("name", _advanced_cases())
def test_port_advanced_matches_circuitscape_golden(name):
    a = np.load(GOLD / "advanced_golden.npz")
    s = np.nan_to_num(a[f"{name}/source"], nan=0.0)
    gr = np.nan_to_num(a[f"{name}/ground"], nan=0.0)
    cur, _ = oracle.advanced(np.nan_to_num(a[f"{name}/conductance"], nan=0.0), s, gr, bool(a[f"{name}/four"]))
    chol = a[f"{name}/current_cholmod"]
    np.testing.assert_array_equal(cur != 0, chol != 0)
    np.testing.assert_allclose(cur, chol, rtol=1e-9, atol=1e-12 * chol.max())


def test_advanced_known_answers():
    # advanced.py:106-123 of the reference: one amp on the left of a 3 x 5 grid, grounded on the right
    g = np.ones((3, 5))
    s = np.zeros((3, 5))
    s[1, 0] = 1.0
    gr = np.zeros((3, 5))
    gr[1, 4] = np.inf
    cur, volt = oracle.advanced(g, s, gr)
    np.testing.assert_array_equal(volt.round(3), [[0.716, 0.615, 0.444, 0.272, 0.172],
                                                   [0.887, 0.615, 0.444, 0.272, 0.],
                                                   [0.716, 0.615, 0.444, 0.272, 0.172]])
    np.testing.assert_array_equal(cur.round(3), [[0.172, 0.293, 0.293, 0.293, 0.172],
                                                  [1., 0.414, 0.414, 0.414, 1.],
                                                  [0.172, 0.293, 0.293, 0.293, 0.172]])
    # tests/test_circuit.py:41-59: two cells, a chain, a diagonal-only pair
    cur, volt = oracle.advanced(np.array([[1.0, 1.0]]), np.array([[1.0, 0.0]]), np.array([[0.0, np.inf]]))
    np.testing.assert_allclose(cur, [[1.0, 1.0]], rtol=1e-14)
    cur, volt = oracle.advanced(np.array([[1.0, 3.0, 2.0]]), np.array([[2.0, 0, 0]]), np.array([[0, 0, np.inf]]))
    np.testing.assert_allclose(volt, [[2 / 2.5 + 2 / 2, 2 / 2.5, 0]], rtol=1e-13)
    g = np.array([[1.0, np.nan], [np.nan, 1.0]])
    cur, volt = oracle.advanced(np.nan_to_num(g), np.array([[1.0, 0], [0, 0]]), np.array([[0, 0], [0, np.inf]]))
    np.testing.assert_allclose(volt[0, 0], np.sqrt(2), rtol=1e-13)
    cur, volt = oracle.advanced(np.nan_to_num(g), np.array([[1.0, 0], [0, 0]]), np.array([[0, 0], [0, np.inf]]),
                                four=True)
    np.testing.assert_array_equal(cur, 0)
    # finite grounds split the current (tests/test_circuit.py:99-104)
    cur, _ = oracle.advanced(np.ones((1, 3)), np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 1.0]]))
    np.testing.assert_allclose(cur, [[0.5, 1.0, 0.5]], rtol=1e-13)


def test_series_weights_known_answer():
    # resistor series (circuitscape.cpp:30-33): conductances 1 and 3 in series -> 1 / ((1 + 1/3) / 2) = 1.5
    cur, volt = oracle.advanced(np.array([[1.0, 3.0]]), np.array([[1.0, 0.0]]), np.array([[0.0, np.inf]]),
                                series=True)
    np.testing.assert_allclose(volt[0, 0], 1 / 1.5, rtol=1e-13)


def test_gap_example():
    # omniscape.py:286-302 of the reference: current concentrates in the gap of a barrier
    r = np.ones((30, 30))
    r[:, 14:16] = 20
    r[10:20, 14:16] = 1
    out = oracle.omniscape(r, 6, flow_potential=True, normalized_current=True)
    assert list(k for k in out if k != "attrs") == ["cum_currmap", "normalized_cum_currmap", "flow_potential"]
    assert round(float(out["cum_currmap"][15, 14]), 2) == 5.16
    assert round(float(out["cum_currmap"][2, 14]), 2) == 1.55


def test_correction_factors():
    # tests/test_omniscape.py:103-110 of the reference
    np.testing.assert_array_equal(oracle.correction(4, 1, 1, False, 50, 50), 1.0)
    c = oracle.correction(6, 2, 5, False, 50, 50)
    assert c.shape == (17, 17)
    np.testing.assert_allclose(c, c.T, rtol=1e-9)
    np.testing.assert_allclose(c, c[::-1, :], rtol=1e-9)
    assert np.all(c > 0)
    if oracle.REF_AVAILABLE:
        np.testing.assert_allclose(c, oracle.ref_correction(6, 2, 5, False, 50, 50), rtol=1e-11)


def test_single_target_is_one_advanced_solve():
    # tests/test_omniscape.py:28-47 of the reference, on the oracle
    r = _map(2, (15, 15))
    r[np.isnan(r)] = 1.0
    s = np.zeros(r.shape)
    s[7, 7] = 1.0
    s[5, 9] = 2.0
    out = oracle.omniscape(r, 4, source=s)
    assert out["attrs"]["n_targets"] == 2
    total = np.zeros(r.shape)
    for (ty, tx), amps, other in [((7, 7), 1.0, (5, 9)), ((5, 9), 2.0, (7, 7))]:
        yy, xx = np.mgrid[:15, :15]
        g = np.where((yy - ty) ** 2 + (xx - tx) ** 2 <= 16, 1 / r, 0.0)
        src = np.zeros(r.shape)
        src[other] = amps
        gr = np.zeros(r.shape)
        gr[ty, tx] = np.inf
        total += oracle.advanced(g, src, gr)[0]
    np.testing.assert_allclose(out["cum_currmap"], total, rtol=1e-12, atol=1e-15)


CASES = [
    dict(radius=5, block_size=1),
    dict(radius=6, block_size=3, buffer=2, flow_potential=True, normalized_current=True),
    dict(radius=4, block_size=5, buffer=1, four_neighbors=True, flow_potential=True),
    dict(radius=7, block_size=3, correct_artifacts=False, resistance_is_conductance=True),
    dict(radius=3, block_size=7, buffer=4),
]


@pytest.mark.skipif(not oracle.REF_AVAILABLE, reason="the reference-compiled oracle was not built here")
@pytest.mark.parametrize("case", range(len(CASES)))
def test_port_matches_reference_build(case):
    kw = dict(CASES[case])
    r = _map(10 + case, (37, 45))
    if kw.get("resistance_is_conductance"):
        r = 1 / r
    a = oracle.omniscape(r, **kw)
    b = oracle.omniscape(r, impl="ref", **kw)
    for k in OUTPUTS:
        if k in b:
            np.testing.assert_array_equal(np.isnan(a[k]), np.isnan(b[k]))
            np.testing.assert_allclose(a[k], b[k], rtol=1e-10, atol=1e-13 * np.nanmax(b[k]))


@pytest.mark.skipif(not oracle.REF_AVAILABLE, reason="the reference-compiled oracle was not built here")
def test_port_matches_reference_build_with_conditions():
    rng = np.random.default_rng(4)
    r = _map(4, (33, 41))
    c1 = rng.uniform(0, 10, r.shape)
    c1f = c1 + rng.normal(0, 1, r.shape)
    c2 = rng.integers(0, 3, r.shape).astype(float)
    c2[rng.random(r.shape) < 0.1] = np.nan
    kw = dict(radius=5, block_size=3, condition1=c1, condition1_future=c1f, compare_to_future="1",
              condition1_lower=-2.0, condition1_upper=1.5, condition2=c2, comparison2="equal")
    a = oracle.omniscape(r, **kw)
    b = oracle.omniscape(r, impl="ref", **kw)
    np.testing.assert_allclose(a["cum_currmap"], b["cum_currmap"], rtol=1e-10,
                               atol=1e-13 * np.nanmax(b["cum_currmap"]))


def test_oracle_adjoint_matches_finite_differences():
    # the FP64 adjoint of the oracle against central differences of the oracle itself
    rng = np.random.default_rng(7)
    r = np.exp(rng.normal(0, 0.7, (24, 26)))
    r[rng.random(r.shape) < 0.04] = np.nan
    s = np.where(rng.random(r.shape) < 0.5, 1.0, 0.0)
    weight = np.zeros(r.shape)
    weight[8:16, 9:18] = 1.0
    J, gr, gs = oracle.omniscape_grad(r, s, weight, 4)
    out = oracle.omniscape(r, 4, source=s, mask_nodata=False)
    assert abs(J - float((weight * out["cum_currmap"]).sum())) <= 1e-12 * abs(J)
    cells = [(y, x) for y, x in zip(rng.integers(2, 22, 12), rng.integers(2, 24, 12)) if not np.isnan(r[y, x])]
    for y, x in cells:
        h = 1e-4 * r[y, x]
        rp, rm = r.copy(), r.copy()
        rp[y, x] += h
        rm[y, x] -= h
        jp = (weight * oracle.omniscape(rp, 4, source=s, mask_nodata=False)["cum_currmap"]).sum()
        jm = (weight * oracle.omniscape(rm, 4, source=s, mask_nodata=False)["cum_currmap"]).sum()
        fd = (jp - jm) / (2 * h)
        assert abs(fd - gr[y, x]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gr).max()), (y, x, fd, gr[y, x])
        if s[y, x] <= 0:  # the positive-source filter is a kink at 0
            continue
        h = 1e-4 * s[y, x]
        sp, sm = s.copy(), s.copy()
        sp[y, x] += h
        sm[y, x] -= h
        jp = (weight * oracle.omniscape(r, 4, source=sp, mask_nodata=False)["cum_currmap"]).sum()
        jm = (weight * oracle.omniscape(r, 4, source=sm, mask_nodata=False)["cum_currmap"]).sum()
        fd = (jp - jm) / (2 * h)
        assert abs(fd - gs[y, x]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gs).max()), (y, x, fd, gs[y, x])
