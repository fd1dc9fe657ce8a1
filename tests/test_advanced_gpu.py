"""The advanced mode on the GPU (``lsb_rasters``): one launch solves a batch of independent rasters.

* the 6 Circuitscape advanced-mode CHOLMOD goldens (islands, four neighbours, finite grounds, several components,
  a window) at the reference's bar, for both solvers, in one batch;
* the reference's known answers (advanced.py:106-123 and tests/test_circuit.py:41-59);
* random rasters of different shapes with several components, finite and direct grounds, signed sources and
  sources on grounded cells, against the oracle's restatement of grid.cpp:73-210: voltages to 1e-9 of the largest,
  currents to 1e-9 relative or 2e-8 of the largest (signed sources put some branch currents within rounding of the
  1e-8 threshold, where leaving one out or not moves a node's current by up to 1e-8 of the largest);
* rasters of the 4096-raster workload (sides 64-512, log-uniform resistance in [1, 1000], one unit source, one
  direct ground, 4 neighbours): small ones against the oracle; all of them by Kirchhoff's law (1 A at the source
  and the ground up to the branches under the threshold, a relative FP64 residual of the node equations below
  1e-10 computed here in numpy).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
SOLVERS = ["fp32-refine", "fp64"]


@pytest.fixture(scope="module")
def lsb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import landschaft_b200
    return landschaft_b200


def _golden():
    a = np.load(GOLD / "advanced_golden.npz")
    names = sorted({k.split("/")[0] for k in a.files})
    return a, names


@pytest.mark.parametrize("solver", SOLVERS)
def test_goldens_in_one_batch(lsb, solver):
    a, names = _golden()
    for four in (False, True):
        sel = [n for n in names if bool(a[f"{n}/four"]) == four]
        if not sel:
            continue
        res = lsb.advanced_batch([(a[f"{n}/conductance"], a[f"{n}/source"], a[f"{n}/ground"]) for n in sel],
                                 four_neighbors=four, solver=solver)
        for n, r in zip(sel, res):
            chol = a[f"{n}/current_cholmod"]
            np.testing.assert_array_equal(r.current != 0, chol != 0, err_msg=n)
            np.testing.assert_allclose(r.current, chol, rtol=1e-9, atol=1e-12 * chol.max(), err_msg=n)


def test_known_answers(lsb):
    g = np.ones((3, 5))
    s = np.zeros((3, 5))
    s[1, 0] = 1.0
    gr = np.zeros((3, 5))
    gr[1, 4] = np.inf
    r = lsb.advanced(g, s, gr)
    np.testing.assert_array_equal(r.voltage.round(3), [[0.716, 0.615, 0.444, 0.272, 0.172],
                                                       [0.887, 0.615, 0.444, 0.272, 0.],
                                                       [0.716, 0.615, 0.444, 0.272, 0.172]])
    np.testing.assert_array_equal(r.current.round(3), [[0.172, 0.293, 0.293, 0.293, 0.172],
                                                       [1., 0.414, 0.414, 0.414, 1.],
                                                       [0.172, 0.293, 0.293, 0.293, 0.172]])
    r = lsb.advanced(np.array([[1.0, 3.0, 2.0]]), np.array([[2.0, 0, 0]]), np.array([[0, 0, np.inf]]))
    np.testing.assert_allclose(r.voltage, [[2 / 2.5 + 2 / 2, 2 / 2.5, 0]], rtol=1e-12)
    g = np.array([[1.0, np.nan], [np.nan, 1.0]])
    r = lsb.advanced(g, np.array([[1.0, 0], [0, 0]]), np.array([[0, 0], [0, np.inf]]))
    np.testing.assert_allclose(r.voltage[0, 0], np.sqrt(2), rtol=1e-12)
    assert np.isnan(r.voltage[0, 1]) and np.isnan(r.voltage[1, 0])
    r = lsb.advanced(g, np.array([[1.0, 0], [0, 0]]), np.array([[0, 0], [0, np.inf]]), four_neighbors=True)
    np.testing.assert_array_equal(r.current, 0)  # no component has both a source and a ground
    np.testing.assert_array_equal(r.voltage[[0, 1], [0, 1]], 0)


def test_validation(lsb):
    g = np.ones((4, 4))
    with pytest.raises(ValueError, match="same shape"):
        lsb.advanced(g, np.zeros((4, 5)), np.zeros((4, 4)))
    with pytest.raises(ValueError, match="finite"):
        lsb.advanced(np.full((4, 4), np.inf), np.zeros((4, 4)), np.zeros((4, 4)))
    with pytest.raises(ValueError, match="negative"):
        lsb.advanced(g, np.zeros((4, 4)), -np.ones((4, 4)))


def _random_case(seed, shape, four):
    rng = np.random.default_rng(seed)
    g = np.exp(rng.normal(0, 1, shape))
    g[rng.random(shape) < 0.25] = 0.0  # holes: several components, islands
    s = np.where(rng.random(shape) < 0.05, rng.uniform(-1, 2, shape), 0.0)
    gr = np.zeros(shape)
    gr[rng.random(shape) < 0.01] = np.inf
    fin = rng.random(shape) < 0.03
    gr[fin] = rng.uniform(0.1, 3, shape)[fin]
    return g, s, gr


@pytest.mark.parametrize("solver", SOLVERS)
@pytest.mark.parametrize("four", [False, True])
def test_random_batch_matches_the_oracle(lsb, solver, four):
    shapes = [(17, 23), (40, 31), (1, 30), (30, 1), (64, 64), (5, 3), (90, 70)]
    cases = [_random_case(100 + k, sh, four) for k, sh in enumerate(shapes)]
    res = lsb.advanced_batch(cases, four_neighbors=four, solver=solver)
    for (g, s, gr), r in zip(cases, res):
        cur, volt = oracle.advanced(g, s, gr, four)
        np.testing.assert_array_equal(np.isnan(r.voltage), np.isnan(volt))
        top = max(np.abs(cur).max(), 1e-300)
        clear = (np.abs(cur) > 2e-8 * top) | (np.abs(r.current) > 2e-8 * top)
        np.testing.assert_array_equal((r.current != 0)[clear], (cur != 0)[clear])
        np.testing.assert_allclose(r.current, cur, rtol=1e-9, atol=2e-8 * top)
        vt = max(np.nanmax(np.abs(volt)), 1e-300)
        m = ~np.isnan(volt)
        np.testing.assert_allclose(r.voltage[m], volt[m], rtol=0, atol=1e-9 * vt)


def _node_residual(g, s, gr, v):
    """Relative FP64 residual of the node equations (4 neighbours, average conductance, direct grounds fixed)."""
    ny, nx = g.shape
    res = np.zeros_like(v)
    acc = np.zeros_like(v)
    for dy, dx in ((0, 1), (1, 0)):
        a = (slice(0, ny - dy), slice(0, nx - dx))
        b = (slice(dy, ny), slice(dx, nx))
        w = (g[a] + g[b]) / 2
        w[(g[a] <= 0) | (g[b] <= 0)] = 0.0
        f = w * (v[a] - v[b])
        res[a] += f
        res[b] -= f
        acc[a] += np.abs(f)
        acc[b] += np.abs(f)
    free = np.isfinite(gr) & (g > 0)
    r = (s - res)[free]
    return np.abs(r).max() / max(np.abs(s).max(), 1.0)


def test_workload_rasters(lsb):
    from landschaft_b200 import synthetic
    cases = synthetic.advanced_rasters(16, seed=3)
    small = [k for k, (g, _, _) in enumerate(cases) if g.size <= 130 * 130][:2]
    cases += synthetic.advanced_rasters(3, seed=4, side_min=64, side_max=100)
    small += [16, 17, 18]
    res, stats = lsb.advanced_batch(cases, four_neighbors=True, return_stats=True)
    assert stats["n_failed"] == 0 and stats["n_solved"] == len(cases)
    for k, ((g, s, gr), r) in enumerate(zip(cases, res)):
        src, gnd = np.argmax(s), np.argmax(np.isinf(gr))
        # 1 A at both ends, less the branch currents under 1e-8 of the largest that the node current leaves out
        assert abs(r.current.flat[src] - 1.0) < 1e-7 and abs(r.current.flat[gnd] - 1.0) < 1e-7
        assert r.voltage.flat[gnd] == 0.0 and np.all(r.voltage > -1e-9)
        assert _node_residual(g, s, gr, r.voltage) < 1e-10
        if k in small:
            cur, volt = oracle.advanced(g, s, gr, True)
            np.testing.assert_allclose(r.current, cur, rtol=1e-9, atol=1e-9 * cur.max())
            np.testing.assert_allclose(r.voltage, volt, rtol=0, atol=1e-9 * volt.max())
