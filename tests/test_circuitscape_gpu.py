"""Circuitscape pairwise mode on the GPU (lsb_graph_pairs) against Circuitscape's goldens and the oracle."""

from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

from landschaft_b200 import _native as N
from landschaft_b200 import circuitscape as cs

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))
import circuitscape_oracle as O  # noqa: E402
from test_circuitscape_cpu import (ADVANCED_CASES, ALL_TO_ONE_CASES, CS, ONE_TO_ALL_CASES, POINT_CASES,  # noqa
                                   REGION_CASES, check_advanced, check_against_golden, check_one_to_all, ini_path,
                                   random_case)

pytestmark = pytest.mark.gpu


@pytest.fixture
def in_cs(monkeypatch):
    monkeypatch.chdir(CS)


@pytest.mark.parametrize("pair_solver", ["auto", "graph"])
@pytest.mark.parametrize("name", POINT_CASES + REGION_CASES)
def test_pairwise_matches_circuitscape(name, pair_solver, in_cs):
    r = cs.circuitscape_ini(ini_path(name), write_outputs=False, pair_solver=pair_solver)
    check_against_golden(name, r.resistances, r.cum_current, r.max_current, r.maps)
    assert r.stats.failures == 0 and r.stats.jobs > 0


def test_docstring_example():
    resistance = np.ones((10, 10))
    resistance[:, 5] = 10
    points = np.zeros((10, 10), dtype=int)
    points[1, 1], points[8, 1], points[5, 8] = 1, 2, 3
    r = cs.circuitscape_pairwise(resistance, points, cum_map=True)
    np.testing.assert_array_equal(r.resistances.round(4), [[0.0, 1.0, 2.0, 3.0], [1.0, 0.0, 0.8515, 0.8567],
                                                          [2.0, 0.8515, 0.0, 0.8409], [3.0, 0.8567, 0.8409, 0.0]])
    assert r.cum_current.shape == (10, 10)


def oracle_pairwise(g, poly, pm, avg, four, opts, excluded_ids=frozenset()):
    G = O.raster_graph(g, poly, avg, four)
    fp = cs._points_from_map(pm)
    rows, cols = fp.cells
    nodes = np.array([G["nodemap"][r * g.shape[1] + c] for r, c in zip(rows, cols)], dtype=np.int64)
    n = len(fp.ids)
    ex = np.array([[(int(fp.ids[a]), int(fp.ids[b])) in excluded_ids for b in range(n)] for a in range(n)],
                  dtype=bool)
    maps = {}

    def emit(ci, cj, vmap, cmap):
        key = (int(fp.ids[ci]), int(fp.ids[cj]))
        if vmap is not None:
            maps[("voltage", *key)] = vmap.reshape(g.shape)
        if cmap is not None:
            maps[("current", *key)] = cmap.reshape(g.shape)

    R, cum, mx = O.pairwise(G, g, nodes, ex, opts, emit)
    return R, cum, mx, maps


@pytest.mark.parametrize("pair_solver", ["auto", "graph"])
@pytest.mark.parametrize("seed", range(6))
def test_random_rasters_match_the_oracle(seed, pair_solver):
    rng = np.random.default_rng(100 + seed)
    ny, nx = (int(v) for v in rng.integers(8, 40, 2))
    g, poly = random_case(rng, ny, nx, seed % 2 == 0)
    pm = np.zeros((ny, nx))
    cells = rng.choice(ny * nx, size=6, replace=False)
    pm.flat[cells] = rng.permutation(np.arange(1, 7))
    avg, four = bool(seed & 1), bool(seed & 2)
    flags = dict(voltage_maps=True, current_maps=True, max_map=True,
                 set_focal_node_currents_to_zero=seed == 3, set_null_currents_to_nodata=seed == 4,
                 set_null_voltages_to_nodata=seed == 4, log_transform_maps=seed == 5)
    r = cs.circuitscape_pairwise(g, pm, habitat_is_resistance=False, polygons=poly, four_neighbors=four,
                                 avg_resistances=avg, pair_solver=pair_solver, **flags)
    opts = {"volt_maps": True, "cur_maps": True, "cum": True, "max": True, "focal_zero": seed == 3,
            "null_currents": seed == 4, "null_voltages": seed == 4, "log_transform": seed == 5}
    R, cum, mx, maps = oracle_pairwise(g, poly, pm, avg, four, opts)
    np.testing.assert_allclose(r.resistances[1:, 1:], R, rtol=1e-9, atol=1e-12)
    scale = max(np.abs(cum).max(), 1e-300)
    np.testing.assert_allclose(r.cum_current, cum.reshape(ny, nx), rtol=1e-8, atol=1e-10 * scale)
    np.testing.assert_allclose(r.max_current, mx.reshape(ny, nx), rtol=1e-8, atol=1e-10 * scale)
    assert set(r.maps) == set(maps)
    for k, want in maps.items():
        np.testing.assert_allclose(r.maps[k], want, rtol=1e-8, atol=1e-10 * max(np.abs(want).max(), 1e-300),
                                   err_msg=str(k))


def test_shortcut_matches_full_solves_and_excluded_pairs():
    rng = np.random.default_rng(7)
    g, poly = random_case(rng, 30, 26, True)
    pm = np.zeros((30, 26))
    pm.flat[rng.choice(30 * 26, size=7, replace=False)] = np.arange(1, 8)
    short = cs.circuitscape_pairwise(g, pm, habitat_is_resistance=False, polygons=poly)
    full = cs.circuitscape_pairwise(g, pm, habitat_is_resistance=False, polygons=poly, cum_map=True)
    np.testing.assert_allclose(full.resistances, short.resistances, rtol=1e-9, atol=1e-12)
    R, _, _, _ = oracle_pairwise(g, poly, pm, False, False, {})
    np.testing.assert_allclose(short.resistances[1:, 1:], R, rtol=1e-9, atol=1e-12)
    pairs = cs.IncludedPairs("exclude", np.array([1, 2, 3]), np.array([[0, 1, 0], [1, 0, 0], [0, 0, 0]]))
    ex = cs.circuitscape_pairwise(g, pm, habitat_is_resistance=False, polygons=poly, included_pairs=pairs)
    R, _, _, _ = oracle_pairwise(g, poly, pm, False, False, {}, pairs.excluded())
    np.testing.assert_allclose(ex.resistances[1:, 1:], R, rtol=1e-9, atol=1e-12)
    assert ex.resistances[1, 2] == -1 and ex.resistances[2, 1] == -1


@pytest.mark.parametrize("pair_solver", ["raster", "graph"])
def test_larger_raster_matches_the_oracle(pair_solver):
    # over 8,192 nodes: the kernel runs 512 threads per CTA
    rng = np.random.default_rng(11)
    ny, nx = 112, 96
    g = 10 ** rng.uniform(0, 2, size=(ny, nx))
    g[rng.random((ny, nx)) < 0.1] = 0
    pm = np.zeros((ny, nx))
    pm.flat[rng.choice(ny * nx, size=5, replace=False)] = np.arange(1, 6)
    r = cs.circuitscape_pairwise(g, pm, habitat_is_resistance=False, cum_map=True, max_map=True,
                                 pair_solver=pair_solver)
    R, cum, mx, _ = oracle_pairwise(g, None, pm, False, False, {"cum": True, "max": True})
    np.testing.assert_allclose(r.resistances[1:, 1:], R, rtol=1e-9)
    np.testing.assert_allclose(r.cum_current, cum.reshape(ny, nx), rtol=1e-8, atol=1e-10 * np.abs(cum).max())
    np.testing.assert_allclose(r.max_current, mx.reshape(ny, nx), rtol=1e-8, atol=1e-10 * np.abs(cum).max())


@pytest.mark.parametrize("polygons", [False, True])
def test_focal_regions_match_the_oracle(polygons):
    rng = np.random.default_rng(21 + polygons)
    ny, nx = 18, 15
    g, poly = random_case(rng, ny, nx, polygons)
    pm = np.zeros((ny, nx))
    pm.flat[rng.choice(ny * nx, size=9, replace=False)] = np.repeat([1, 2, 3, 4], [3, 2, 3, 1])
    r = cs.circuitscape_pairwise(g, pm, habitat_is_resistance=False, polygons=poly, current_maps=True,
                                 voltage_maps=True, max_map=True)
    fp = cs._points_from_map(pm)
    rows, cols = fp.cells
    cells = [int(a * nx + b) for a, b in zip(rows, cols)]
    maps = {}

    def emit(ci, cj, vmap, cmap):
        key = (ci + 1, cj + 1)
        if vmap is not None:
            maps[("voltage", *key)] = vmap.reshape(ny, nx)
        if cmap is not None:
            maps[("current", *key)] = cmap.reshape(ny, nx)

    opts = {"volt_maps": True, "cur_maps": True, "cum": True, "max": True}
    ids, R, cum, mx = O.pairwise_regions(g, poly, False, False, cells, [int(v) for v in fp.ids],
                                         np.zeros((4, 4), dtype=bool), opts, emit)
    np.testing.assert_array_equal(r.resistances[0, 1:], ids)
    np.testing.assert_allclose(r.resistances[1:, 1:], R, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(r.cum_current, cum.reshape(ny, nx), rtol=1e-8, atol=1e-10 * np.abs(cum).max())
    np.testing.assert_allclose(r.max_current, mx.reshape(ny, nx), rtol=1e-8, atol=1e-10 * np.abs(cum).max())
    assert set(r.maps) == set(maps)
    for k, want in maps.items():
        np.testing.assert_allclose(r.maps[k], want, rtol=1e-8, atol=1e-10 * max(np.abs(want).max(), 1e-300))


def solve_path(w, ground, src, dst, params):
    """lsb_graph_pairs on a path graph 0 - 1 - ... - n-1 with conductances w; returns (rc, volt, cur, stats)."""
    import torch
    lib = N.load()
    n = len(w) + 1
    adj, wt, ptr = [], [], [0]
    for i in range(n):
        for k in (i - 1, i + 1):
            if 0 <= k < n:
                adj.append(k)
                wt.append(w[min(i, k)])
        ptr.append(len(adj))
    diag = np.array([sum(wt[ptr[i]:ptr[i + 1]]) for i in range(n)]) + cs.K_SHIFT
    dev = torch.device("cuda", 0)
    t = lambda a, dt: torch.tensor(np.asarray(a), dtype=dt, device=dev)  # noqa: E731
    d_ptr, d_adj, d_w, d_diag = t(ptr, torch.int64), t(adj, torch.int32), t(wt, torch.float64), t(diag, torch.float64)
    d_src, d_dst = t(src, torch.int32), t(dst, torch.int32)
    nj = len(src)
    volt = torch.empty((nj, n), dtype=torch.float64, device=dev)
    cur = torch.empty_like(volt)
    nb = C.c_size_t(0)
    assert lib.lsb_graph_pairs_workspace_size(n, nj, C.byref(params), C.byref(nb)) == 0
    ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    st = N.GraphStats()
    err = C.create_string_buffer(256)
    rc = lib.lsb_graph_pairs(n, d_ptr.data_ptr(), d_adj.data_ptr(), d_w.data_ptr(), d_diag.data_ptr(), ground, nj,
                             d_src.data_ptr(), d_dst.data_ptr(), C.byref(params), volt.data_ptr(), cur.data_ptr(),
                             ws.data_ptr(), nb.value, C.byref(st), err, len(err),
                             torch.cuda.current_stream().cuda_stream)
    return rc, volt.cpu().numpy(), cur.cpu().numpy(), st, err.value


def test_series_resistors_closed_form():
    w = [2.0, 0.5, 4.0, 1.0]
    rc, volt, cur, st, _ = solve_path(w, 4, [0, 1, 4], [4, 3, 0], N.default_graph_params())
    assert rc == 0 and st.failures == 0 and st.jobs == 3
    np.testing.assert_allclose(volt[0, 4] - volt[0, 0], sum(1 / x for x in w), rtol=1e-12)
    np.testing.assert_allclose(volt[1, 3] - volt[1, 1], 1 / 0.5 + 1 / 4.0, rtol=1e-12)
    np.testing.assert_allclose(volt[2, 0] - volt[2, 4], sum(1 / x for x in w), rtol=1e-12)
    assert volt[0, 0] == 0.0  # relative to the source
    np.testing.assert_allclose(cur[0], np.ones(5), rtol=1e-12)  # a unit current through every node
    np.testing.assert_allclose(cur[1], [0, 1, 1, 1, 0], atol=1e-12)


def test_iteration_cap_reports_failure():
    p = N.default_graph_params()
    p.max_iter = 1
    rc, _, _, st, err = solve_path([1.0] * 30, 30, [0], [15], p)
    assert rc == N.LSB_ERR_NOT_CONVERGED and st.failures == 1 and b"failed" in err
    p = N.default_graph_params()
    rc, _, _, st, _ = solve_path([1.0] * 30, 30, [0, 40], [15, 3], p)  # a node index out of range fails that job
    assert rc == N.LSB_ERR_NOT_CONVERGED and st.failures == 1


# --- advanced, one-to-all and all-to-one (lsb_graph_solve) ---------------------------------------------------------

@pytest.mark.parametrize("problem_solver", ["auto", "graph"])
@pytest.mark.parametrize("ini", ADVANCED_CASES)
def test_advanced_matches_circuitscape(ini, problem_solver, in_cs):
    # the reference's bar, rtol 1e-9
    check_advanced(Path(ini).stem, cs.circuitscape_ini(ini, write_outputs=False, problem_solver=problem_solver))


@pytest.mark.parametrize("problem_solver", ["auto", "graph"])
@pytest.mark.parametrize("ini", ONE_TO_ALL_CASES + ALL_TO_ONE_CASES)
def test_one_to_all_matches_circuitscape(ini, problem_solver, in_cs):
    # the reference's bar is 1e-11 for its direct solver; the GPU's iterative solve is held to 1e-9
    check_one_to_all(Path(ini).stem, cs.circuitscape_ini(ini, write_outputs=False, problem_solver=problem_solver), rtol=1e-9)


@pytest.mark.parametrize("policy", cs.POLICIES)
def test_random_advanced_matches_the_oracle(policy):
    rng = np.random.default_rng(40 + cs.POLICIES.index(policy))
    ny, nx = 23, 19
    g, poly = random_case(rng, ny, nx, True)
    src = np.where(rng.random((ny, nx)) < 0.05, rng.normal(size=(ny, nx)), 0.0)
    gnd = np.where(rng.random((ny, nx)) < 0.05, rng.choice([0.0, 0.3, 4.0], (ny, nx)), cs.NODATA)
    kw = dict(habitat_is_resistance=False, polygons=poly, remove_src_or_gnd=policy)
    r = cs.circuitscape_advanced(g, src, gnd, **kw)
    gr = np.where(gnd == cs.NODATA, 0.0, np.divide(1.0, gnd, out=np.full_like(gnd, np.inf), where=gnd != 0))
    want = cs._advanced(g, poly, src, gr, False, False, policy, False, False, O.multi_advanced)
    assert r.maps["solved"] == want.maps["solved"]
    np.testing.assert_array_equal(r.nodemap, want.nodemap)
    for ours, ref in ((r.voltage, want.voltage), (r.current, want.current)):
        np.testing.assert_allclose(ours, ref, rtol=1e-9, atol=1e-11 * max(np.abs(ref).max(), 1e-300))


@pytest.mark.parametrize("all_to_one", [False, True])
def test_one_to_all_api_matches_the_oracle(all_to_one):
    rng = np.random.default_rng(50 + all_to_one)
    ny, nx = 20, 24
    g, poly = random_case(rng, ny, nx, True)
    pm = np.zeros((ny, nx))
    pm.flat[rng.choice(ny * nx, size=6, replace=False)] = np.arange(1, 7)
    flags = dict(habitat_is_resistance=False, polygons=poly, voltage_maps=True, current_maps=True, max_map=True)
    r = cs.circuitscape_one_to_all(g, pm, all_to_one=all_to_one, **flags)
    maps = {}

    def emit(n, volt, cur):
        if volt is not None:
            maps[("voltage", n)] = volt
        if cur is not None:
            maps[("current", n)] = cur

    opts = {"volt_maps": True, "cur_maps": True, "cum": True, "max": True, "focal_zero": False}
    want = cs._one_to_all(g, poly, cs._points_from_map(pm), None, None, not all_to_one, False, False, opts, emit,
                          O.multi_advanced)
    np.testing.assert_allclose(r.resistances, want.resistances, rtol=1e-9, atol=1e-12)
    scale = np.abs(want.cum_current).max()
    np.testing.assert_allclose(r.cum_current, want.cum_current, rtol=1e-9, atol=1e-11 * scale)
    np.testing.assert_allclose(r.max_current, want.max_current, rtol=1e-9, atol=1e-11 * scale)
    assert set(r.maps) == set(maps)
    for k, v in maps.items():
        np.testing.assert_allclose(r.maps[k], v, rtol=1e-9, atol=1e-11 * max(np.abs(v).max(), 1e-300))


def test_graph_solve_closed_form():
    # a path 0 - 1 - 2 - 3 with conductances w: a unit source at 0 and a finite ground of conductance 0.5 at 3
    # (voltages sum 1/w + 1/0.5 down the path); a second job with a direct ground at 3 instead
    import torch
    lib = N.load()
    w = [2.0, 0.5, 4.0]
    n = 4
    adj, wt, ptr = [], [], [0]
    for i in range(n):
        for k in (i - 1, i + 1):
            if 0 <= k < n:
                adj.append(k)
                wt.append(w[min(i, k)])
        ptr.append(len(adj))
    diag = np.array([sum(wt[ptr[i]:ptr[i + 1]]) for i in range(n)]) + cs.K_SHIFT
    dev = torch.device("cuda", 0)
    t = lambda a, dt: torch.tensor(np.asarray(a), dtype=dt, device=dev)  # noqa: E731
    args = [t(ptr, torch.int64), t(adj, torch.int32), t(wt, torch.float64), t(diag, torch.float64)]
    lists = [t([0, 1, 2], torch.int64), t([0, 0], torch.int32), t([1.0, 1.0], torch.float64),
             t([0, 0, 1], torch.int64), t([3], torch.int32), t([0, 1, 1], torch.int64), t([3], torch.int32),
             t([0.5], torch.float64)]
    volt = torch.empty((2, n), dtype=torch.float64, device=dev)
    cur = torch.empty_like(volt)
    p = N.default_graph_params()
    nb = C.c_size_t(0)
    assert lib.lsb_graph_solve_workspace_size(n, 2, C.byref(p), C.byref(nb)) == 0
    ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    st = N.GraphStats()
    err = C.create_string_buffer(256)
    rc = lib.lsb_graph_solve(n, *(a.data_ptr() for a in args), 2, *(a.data_ptr() for a in lists), C.byref(p),
                             volt.data_ptr(), cur.data_ptr(), ws.data_ptr(), nb.value, C.byref(st), err, len(err),
                             torch.cuda.current_stream().cuda_stream)
    assert rc == 0 and st.failures == 0, err.value
    v, c = volt.cpu().numpy(), cur.cpu().numpy()
    np.testing.assert_allclose(v[0], [1 / 2 + 1 / 0.5 + 1 / 4 + 2, 1 / 0.5 + 1 / 4 + 2, 1 / 4 + 2, 2], rtol=1e-12)
    np.testing.assert_allclose(c[0], np.ones(4), rtol=1e-12)  # the finite ground's current counts at node 3
    np.testing.assert_allclose(v[1], [1 / 2 + 1 / 0.5 + 1 / 4, 1 / 0.5 + 1 / 4, 1 / 4, 0.0], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(c[1], np.ones(4), rtol=1e-12)


def test_large_advanced_matches_the_oracle():
    # over 8,192 nodes (512 threads per CTA), finite and direct grounds, several sources
    rng = np.random.default_rng(61)
    ny, nx = 104, 96
    g = 10 ** rng.uniform(0, 2, size=(ny, nx))
    g[rng.random((ny, nx)) < 0.05] = 0
    src = np.zeros((ny, nx))
    src.flat[rng.choice(ny * nx, 5, replace=False)] = rng.uniform(0.5, 2.0, 5)
    gr = np.zeros((ny, nx))
    gr.flat[rng.choice(ny * nx, 3, replace=False)] = [np.inf, 0.7, 3.0]
    r = cs._advanced(g, None, src, gr, False, False, "keepall", False, False, cs.multi_advanced)
    want = cs._advanced(g, None, src, gr, False, False, "keepall", False, False, O.multi_advanced)
    for ours, ref in ((r.voltage, want.voltage), (r.current, want.current)):
        np.testing.assert_allclose(ours, ref, rtol=1e-9, atol=1e-11 * np.abs(ref).max())


@pytest.mark.parametrize("all_to_one", [False, True])
def test_plain_grid_problems_on_the_raster_route(all_to_one):
    # no polygons: the problems qualify for the raster solver; "raster" forces it, the oracle checks it
    rng = np.random.default_rng(70 + all_to_one)
    ny, nx = 30, 34
    g = np.exp(rng.normal(size=(ny, nx)))
    g[rng.random((ny, nx)) < 0.15] = 0
    pm = np.zeros((ny, nx))
    pm.flat[rng.choice(ny * nx, size=5, replace=False)] = np.arange(1, 6)
    flags = dict(habitat_is_resistance=False, voltage_maps=True, current_maps=True, max_map=True)
    r = cs.circuitscape_one_to_all(g, pm, all_to_one=all_to_one, problem_solver="raster", **flags)
    maps = {}

    def emit(n, volt, cur):
        if volt is not None:
            maps[("voltage", n)] = volt
        if cur is not None:
            maps[("current", n)] = cur

    opts = {"volt_maps": True, "cur_maps": True, "cum": True, "max": True, "focal_zero": False}
    want = cs._one_to_all(g, None, cs._points_from_map(pm), None, None, not all_to_one, False, False, opts, emit,
                          O.multi_advanced)
    np.testing.assert_allclose(r.resistances, want.resistances, rtol=1e-9, atol=1e-12)
    scale = np.abs(want.cum_current).max()
    np.testing.assert_allclose(r.cum_current, want.cum_current, rtol=1e-9, atol=1e-11 * scale)
    assert set(r.maps) == set(maps)
    for k, v in maps.items():
        np.testing.assert_allclose(r.maps[k], v, rtol=1e-9, atol=1e-11 * max(np.abs(v).max(), 1e-300))


def test_plain_grid_advanced_with_finite_grounds_on_the_raster_route():
    rng = np.random.default_rng(80)
    ny, nx = 40, 36
    g = 10 ** rng.uniform(0, 2, size=(ny, nx))
    g[rng.random((ny, nx)) < 0.1] = 0
    src = np.zeros((ny, nx))
    src.flat[rng.choice(ny * nx, 4, replace=False)] = [1.0, 2.0, 0.5, 1.5]
    gr = np.zeros((ny, nx))
    cand = np.flatnonzero(src.ravel() == 0)
    gr.flat[rng.choice(cand, 3, replace=False)] = [np.inf, 0.7, 3.0]
    r = cs._advanced(g, None, src, gr, False, False, "keepall", False, False,
                     lambda *a: cs.multi_advanced(*a, problem_solver="raster"))
    want = cs._advanced(g, None, src, gr, False, False, "keepall", False, False, O.multi_advanced)
    assert r.maps["solved"] == want.maps["solved"]
    for ours, ref in ((r.voltage, want.voltage), (r.current, want.current)):
        np.testing.assert_allclose(ours, ref, rtol=1e-9, atol=1e-11 * np.abs(ref).max())


def test_pairwise_ini_writes_outputs(tmp_path, in_cs):
    src = CS / "input/raster/pairwise/1/sgVerify1.ini"
    out = cs.parse_config(src)["output_file"]
    ini = tmp_path / "run.ini"
    ini.write_text(src.read_text().replace(out, (tmp_path / "pw.out").as_posix()))
    r = cs.circuitscape_ini(ini)
    np.testing.assert_array_equal(np.loadtxt(tmp_path / "pw_resistances.out"), r.resistances)
    three = np.loadtxt(tmp_path / "pw_resistances_3columns.out")
    n = len(r.resistances) - 1
    assert three.shape == (n * (n - 1) // 2, 3)
    np.testing.assert_array_equal(cs.read_raster(tmp_path / "pw_cum_curmap.asc")[0], r.cum_current)
    assert (tmp_path / "pw_curmap_1_2.asc").exists() and r.maps == {}
