"""Circuitscape pairwise mode, host side: the oracle against Circuitscape's goldens, the package's node graph
against the oracle's, the readers, and the C ABI's argument checks (no GPU)."""

from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

from landschaft_b200 import _native as N
from landschaft_b200 import circuitscape as cs

ROOT = Path(__file__).resolve().parents[1]
CS = ROOT / "tests" / "golden" / "circuitscape"
sys.path.insert(0, str(ROOT / "oracle"))
import circuitscape_oracle as O  # noqa: E402

POINT_CASES = ["sgVerify1", "sgVerify2", "sgVerify4", "sgVerify7", "sgVerify12", "sgVerify13", "sgVerify14", "sgVerify15",
               "sgVerify16", "sgVerify17"]
REGION_CASES = ["sgVerify3", "sgVerify5", "sgVerify6", "sgVerify8", "sgVerify9", "sgVerify10", "sgVerify11"]


def ini_path(name):
    return f"input/raster/pairwise/{name.removeprefix('sgVerify')}/{name}.ini"


@pytest.fixture
def in_cs(monkeypatch):
    # the INI files hold paths relative to Circuitscape's test directory
    monkeypatch.chdir(CS)


def check_against_golden(name, res, cum, mx, maps):
    z = np.load(CS / "pairwise.npz")
    ref = z[f"{name}/result.txt"]
    np.testing.assert_allclose(res, ref, rtol=1e-8, atol=1e-12)
    for key, ours in (("cum_curmap.asc", cum), ("max_curmap.asc", mx)):
        if f"{name}/{key}" in z.files:
            want = z[f"{name}/{key}"]
            np.testing.assert_allclose(ours, want, rtol=1e-9, atol=1e-11 * np.abs(want).max())
    theirs = {k.split("/")[1][:-4] for k in z.files if k.startswith(name + "/")
              and k.split("/")[1].startswith(("curmap_", "voltmap_"))}
    assert set(maps) == theirs
    for kind in theirs:
        want = z[f"{name}/{kind}.asc"]
        np.testing.assert_allclose(maps[kind], want, rtol=1e-9, atol=1e-11 * max(np.abs(want).max(), 1e-300))


@pytest.mark.parametrize("name", POINT_CASES + REGION_CASES)
def test_oracle_matches_circuitscape(name, in_cs):
    check_against_golden(name, *O.pairwise_ini(ini_path(name)))


def random_case(rng, ny, nx, polygons):
    g = np.exp(rng.normal(size=(ny, nx)))
    g[rng.random((ny, nx)) < 0.2] = 0
    poly = None
    if polygons:
        poly = np.zeros((ny, nx), dtype=np.int64)
        for pid in range(1, 4):
            y, x = rng.integers(0, ny), rng.integers(0, nx)
            poly[y:y + rng.integers(1, 4), x:x + rng.integers(1, 4)] = pid
    return g, poly


@pytest.mark.parametrize("avg", [False, True])
@pytest.mark.parametrize("four", [False, True])
def test_node_graph_matches_the_oracle(avg, four):
    rng = np.random.default_rng(1 + 2 * avg + four)
    for trial in range(25):
        ny, nx = (int(v) for v in rng.integers(1, 14, 2))
        g, poly = random_case(rng, ny, nx, trial % 2 == 1)
        a = cs.raster_graph(g, poly, avg, four)
        b = O.raster_graph(g, poly, avg, four)
        assert a.n_nodes == b["n_nodes"] and a.n_comp == b["n_comp"]
        np.testing.assert_array_equal(a.nodemap, b["nodemap"])
        np.testing.assert_array_equal(a.comp, b["comp"])
        np.testing.assert_array_equal(a.adj, np.array([r for row in b["rows"] for r, _ in row], dtype=np.int32))
        np.testing.assert_array_equal(a.w, np.array([w for row in b["rows"] for _, w in row]))
        np.testing.assert_array_equal(a.degree, b["degree"])


def test_merged_nodes_and_zero_weight_edges():
    # a non-habitat cell inside a polygon joins its node; with average resistances its edges weigh 0 and do not
    # connect components
    g = np.array([[1.0, 0.0, 1.0], [0.0, 0.0, 0.0], [1.0, 0.0, 1.0]])
    poly = np.array([[1, 1, 0], [0, 0, 0], [0, 0, 0]])
    a = cs.raster_graph(g, poly, True, True)
    assert a.n_nodes == 4 and a.nodemap[0] == a.nodemap[1]
    b = cs.raster_graph(g, poly, False, True)
    assert a.n_comp == 4 and b.n_comp == 3  # average conductance joins (0,2) through the merged cell


def test_readers(in_cs):
    assert cs.file_type("input/raster/pairwise/2/cellmap.asc") == "aagrid"
    assert cs.file_type("input/raster/pairwise/13/include_matrix.txt") == "pairs_aagrid"
    assert cs.file_type("input/raster/pairwise/17/pairs_to_include.txt") == "pairs"
    assert cs.file_type("input/raster/pairwise/7/points5x5.txt") == "list"
    assert cs.file_type("input/raster/pairwise/1/polygons.tif") == "geotiff"
    cells, meta = cs.read_raster("input/raster/pairwise/15/cellmap.asc.gz")
    assert cells.shape == (meta.nrows, meta.ncols) == (10, 10)
    p = cs.read_included_pairs("input/raster/pairwise/17/pairs_to_include.txt")
    assert p.mode == "include" and 1 in p.ids
    tif, meta = cs.read_raster("input/raster/pairwise/1/polygons.tif")
    asc, _ = cs.read_raster("input/raster/pairwise/1/polygons.asc")
    assert (meta.nrows, meta.ncols) == (10, 10)
    np.testing.assert_array_equal(tif, asc)
    tif, meta = cs.read_raster("input/raster/pairwise/10/cellmap7.tif")
    asc, meta2 = cs.read_raster("input/raster/pairwise/11/cellmap7.asc")
    assert (meta.nrows, meta.ncols) == (meta2.nrows, meta2.ncols)


def test_region_polymap_matches_the_oracle():
    rng = np.random.default_rng(5)
    for trial in range(30):
        ny, nx = (int(v) for v in rng.integers(3, 12, 2))
        poly = None
        if trial % 2:
            poly = np.zeros((ny, nx), dtype=np.int64)
            for pid in range(1, 4):
                y, x = rng.integers(0, ny), rng.integers(0, nx)
                poly[y:y + 3, x:x + 2] = pid
        cells = rng.choice(ny * nx, size=7, replace=False).astype(np.int64)
        ids = np.sort(rng.integers(1, 4, size=7))
        for a, b in ((1, 2), (1, 3), (2, 3)):
            np.testing.assert_array_equal(cs.region_polymap(poly, ny * nx, cells, ids, a, b),
                                          O.region_polymap(poly, ny * nx, list(cells), list(ids), a, b))


def test_ini_errors(tmp_path):
    ini = tmp_path / "a.ini"
    ini.write_text("[Options]\nscenario = one-to-many\n")
    with pytest.raises(ValueError, match="scenario"):
        cs.circuitscape_ini(ini)
    ini.write_text("[Options]\ndata_type = network\nscenario = pairwise\n")
    with pytest.raises(NotImplementedError):
        cs.circuitscape_ini(ini)
    ini.write_text("[Options]\nscenario = advanced\nremove_src_or_gnd = rmvsome\n")
    with pytest.raises(ValueError):
        cs.circuitscape_ini(ini)
    ini.write_text("[Options]\nscenario = pairwise\nuse_polygons = maybe\nhabitat_file = x.asc\n")
    with pytest.raises(FileNotFoundError):
        cs.circuitscape_ini(ini)


def test_graph_abi_argument_checks():
    lib = N.load()
    p = N.default_graph_params()
    assert (p.tol, p.accept, p.max_iter, p.max_ctas) == (1e-14, 1e-9, 0, 0)
    nb = C.c_size_t(0)
    assert lib.lsb_graph_pairs_workspace_size(0, 1, C.byref(p), C.byref(nb)) == N.LSB_ERR_ARGUMENT
    assert lib.lsb_graph_pairs_workspace_size(10, -1, C.byref(p), C.byref(nb)) == N.LSB_ERR_ARGUMENT
    assert lib.lsb_graph_pairs_workspace_size(1000, 7, C.byref(p), C.byref(nb)) == N.LSB_OK
    assert nb.value >= 7 * 3 * 1000 * 8
    err = C.create_string_buffer(256)
    st = N.GraphStats()
    # ground out of range, and an empty job list (returns before touching any device memory)
    rc = lib.lsb_graph_pairs(5, None, None, None, None, 5, 1, None, None, C.byref(p), None, None, None, 0,
                             C.byref(st), err, len(err), None)
    assert rc == N.LSB_ERR_ARGUMENT and b"ground" in err.value
    rc = lib.lsb_graph_pairs(5, None, None, None, None, 0, 0, None, None, C.byref(p), None, None, None, 0,
                             C.byref(st), err, len(err), None)
    assert rc == N.LSB_OK and st.jobs == 0
    rc = lib.lsb_graph_pairs(5, None, None, None, None, 0, 2, None, None, C.byref(p), None, None, None, 0,
                             C.byref(st), err, len(err), None)
    assert rc == N.LSB_ERR_ARGUMENT


# --- advanced, one-to-all and all-to-one ---------------------------------------------------------------------------

def _mode_cases(scenario):
    return sorted(str(p.relative_to(CS)) for p in (CS / "input" / "raster" / scenario).glob("*/*.ini"))


ADVANCED_CASES = _mode_cases("advanced")
ONE_TO_ALL_CASES = _mode_cases("one_to_all")
ALL_TO_ONE_CASES = _mode_cases("all_to_one")


def check_advanced(name, r, rtol=1e-9):
    """The reference's bar for advanced mode: zero pattern equal, values within rtol (atol 1e-11 of the largest)."""
    z = np.load(CS / "modes.npz")
    checked = 0
    for key, ours in (("voltmap.asc", r.voltage), ("curmap.asc", r.current), ("result.txt", r.voltage)):
        k = f"{name}/{key}"
        if k not in z.files:
            continue
        ref = z[k]
        np.testing.assert_array_equal(ours == 0, ref == 0)
        np.testing.assert_allclose(ours, ref, rtol=rtol, atol=1e-11 * np.abs(ref).max())
        checked += 1
    assert checked >= 2


def check_one_to_all(name, r, rtol=1e-11):
    """The reference's bar for one-to-all / all-to-one (rtol 1e-11 with a direct solver)."""
    z = np.load(CS / "modes.npz")
    np.testing.assert_allclose(r.resistances, z[f"{name}/result.txt"], rtol=rtol, atol=rtol * 1e-2)
    for key, ours in (("cum_curmap.asc", r.cum_current), ("max_curmap.asc", r.max_current)):
        if f"{name}/{key}" in z.files:
            want = z[f"{name}/{key}"]
            np.testing.assert_allclose(ours, want, rtol=rtol, atol=rtol * 0.1 * np.abs(want).max())
    theirs = {k.split("/")[1][:-4] for k in z.files if k.startswith(name + "/")
              and k.split("/")[1].startswith(("curmap_", "voltmap_"))}
    assert set(r.maps) == theirs
    for kind in theirs:
        want = z[f"{name}/{kind}.asc"]
        np.testing.assert_allclose(r.maps[kind], want, rtol=rtol, atol=rtol * 0.1 * max(np.abs(want).max(), 1e-300))


@pytest.mark.parametrize("ini", ADVANCED_CASES)
def test_oracle_matches_circuitscape_advanced(ini, in_cs):
    check_advanced(Path(ini).stem, cs.circuitscape_ini(ini, write_outputs=False, _solver=O.multi_advanced))


@pytest.mark.parametrize("ini", ONE_TO_ALL_CASES + ALL_TO_ONE_CASES)
def test_oracle_matches_circuitscape_one_to_all(ini, in_cs):
    check_one_to_all(Path(ini).stem, cs.circuitscape_ini(ini, write_outputs=False, _solver=O.multi_advanced))


def test_mode_case_counts():
    assert (len(ADVANCED_CASES), len(ONE_TO_ALL_CASES), len(ALL_TO_ONE_CASES)) == (8, 13, 12)


@pytest.mark.parametrize("policy", cs.POLICIES)
def test_node_sums_and_conflicts_match_the_oracle(policy):
    rng = np.random.default_rng(3)
    g, poly = random_case(rng, 11, 9, True)
    graph = cs.raster_graph(g, poly, False, False)
    G = O.raster_graph(g, poly, False, False)
    cells = rng.integers(0, g.size, 30)
    vals = rng.normal(size=30)
    vals[::5] = 0.0
    np.testing.assert_array_equal(cs.node_sums(graph, cells, vals), O.node_sums(G, list(cells), list(vals)))
    src = np.where(rng.random(graph.n_nodes) < 0.3, rng.normal(size=graph.n_nodes), 0.0)
    gnd = np.where(rng.random(graph.n_nodes) < 0.3, rng.choice([0.5, 2.0, np.inf], graph.n_nodes), 0.0)
    for a, b in zip(cs.resolve_conflicts(src, gnd, policy), O.resolve(list(src), list(gnd), policy)):
        np.testing.assert_array_equal(a, np.array(b))


def test_pair_solver_routing():
    g = np.exp(np.random.default_rng(8).normal(size=(9, 7)))
    g[2, 3] = 0
    plain = cs.raster_graph(g, None, False, False)
    assert cs.raster_route(plain) and not plain.merged
    poly = np.zeros(g.shape, dtype=np.int64)
    poly[4:6, 1:3] = 1
    assert cs.raster_graph(g, poly, False, False).merged  # four cells in one node
    lone = np.zeros(g.shape, dtype=np.int64)
    lone[0, 0] = 5
    assert not cs.raster_graph(g, lone, False, False).merged  # a one-cell region is a plain node
    assert not cs.raster_route(cs.raster_graph(g, None, True, False))  # resistor-series weights
    pts = np.array([0, 5])
    ex = np.zeros((2, 2), dtype=bool)
    with pytest.raises(ValueError, match="pair_solver"):
        cs.raster_pairwise(plain, g, pts, ex, cs.PairOptions(), pair_solver="direct")
    with pytest.raises(ValueError, match="plain grid"):
        cs.raster_pairwise(cs.raster_graph(g, poly, False, False), g, pts, ex, cs.PairOptions(),
                           pair_solver="raster")


def test_summed_maps_equal_the_per_pair_maps(monkeypatch):
    # the cum / max maps from the jobs' currents at once are bitwise those of the per-pair additions (the solve is
    # replaced by a deterministic fake, so this runs without a GPU)
    def fake(graph, members, ground, src, dst, want_currents, params, stats, dev):
        r = np.random.default_rng(int(src.sum() * 7 + dst.sum()))
        v = r.normal(size=(len(src), len(members)))
        c = np.abs(r.normal(size=(len(src), len(members))))
        return v, (c if want_currents else None)

    monkeypatch.setattr(cs, "_solve_component", fake)
    rng = np.random.default_rng(0)
    for trial in range(12):
        ny, nx = (int(v) for v in rng.integers(5, 30, 2))
        g = np.exp(rng.normal(size=(ny, nx)))
        g[rng.random((ny, nx)) < 0.3] = 0
        graph = cs.raster_graph(g, None, False, False)
        pts = rng.permutation(np.unique(graph.nodemap[graph.nodemap >= 0])[:7])
        ex = np.zeros((len(pts), len(pts)), dtype=bool)
        if trial % 3 == 0:
            ex[0, 1] = ex[1, 0] = True
        a = cs.raster_pairwise(graph, g, pts, ex, cs.PairOptions(cum=True, max=True), device="cpu",
                               pair_solver="graph")
        b = cs.raster_pairwise(graph, g, pts, ex, cs.PairOptions(cum=True, max=True, cur_maps=True),
                               lambda *x: None, device="cpu", pair_solver="graph")
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_problem_solver_option():
    g = np.exp(np.random.default_rng(9).normal(size=(6, 5)))
    prob = {"src_cells": np.array([0]), "src_vals": np.array([1.0]), "gnd_cells": np.array([29]),
            "gnd_vals": np.array([np.inf]), "check_cell": -1}
    with pytest.raises(ValueError, match="problem_solver"):
        cs.multi_advanced(g, None, False, False, [prob], "keepall", problem_solver="direct")
    poly = np.zeros(g.shape, dtype=np.int64)
    poly[2:4, 1:3] = 1
    with pytest.raises(ValueError, match="plain grid"):  # merged nodes: not for the raster solver
        cs.multi_advanced(g, poly, False, False, [prob], "keepall", problem_solver="raster")


@pytest.mark.parametrize("four", [False, True])
def test_lite_graph_equals_the_full_graph(four):
    rng = np.random.default_rng(12 + four)
    for trial in range(60):
        ny, nx = (int(v) for v in rng.integers(1, 25, 2))
        g = np.exp(rng.normal(size=(ny, nx)))
        g[rng.random((ny, nx)) < rng.uniform(0, 0.6)] = 0
        a = cs.raster_graph(g, None, False, four)
        b = cs.raster_graph(g, None, False, four, lite=True)
        assert b.ptr is None and (a.n_nodes, a.n_comp) == (b.n_nodes, b.n_comp)
        np.testing.assert_array_equal(a.nodemap, b.nodemap)
        np.testing.assert_array_equal(a.comp, b.comp)
    poly = np.zeros((5, 5), dtype=np.int64)
    poly[1:3, 1:3] = 1
    assert cs.raster_graph(np.ones((5, 5)), poly, False, four, lite=True).ptr is not None  # merged: built in full
    assert cs.raster_graph(np.ones((5, 5)), None, True, four, lite=True).ptr is not None  # series weights: in full


def test_wide_rasters_fall_back_to_the_full_graph(monkeypatch):
    # over 1024 cells wide: "auto" cannot use the raster solver, so the lite graph is rebuilt in full for the
    # node-graph kernel; the results equal those of pair_solver="graph" (the solve is a deterministic fake)
    seen = []

    def fake(graph, members, ground, src, dst, want_currents, params, stats, dev):
        seen.append(graph.ptr is not None)
        r = np.random.default_rng(int(src.sum() * 3 + dst.sum()))
        return r.normal(size=(len(src), len(members))), np.abs(r.normal(size=(len(src), len(members))))

    monkeypatch.setattr(cs, "_solve_component", fake)
    rng = np.random.default_rng(4)
    g = np.exp(rng.normal(size=(3, 1100)))
    pm = np.zeros(g.shape)
    pm[0, 5], pm[2, 600], pm[1, 1090] = 1, 2, 3
    a = cs.circuitscape_pairwise(g, pm, habitat_is_resistance=False, cum_map=True, device="cpu")
    b = cs.circuitscape_pairwise(g, pm, habitat_is_resistance=False, cum_map=True, device="cpu", pair_solver="graph")
    assert seen and all(seen)
    np.testing.assert_array_equal(a.resistances, b.resistances)
    np.testing.assert_array_equal(a.cum_current, b.cum_current)


def test_one_to_all_ini_writes_outputs(tmp_path, in_cs):
    # as Circuitscape writes them: the configuration, the cum map and every point's maps, read back bitwise
    src = CS / "input/raster/one_to_all/1/oneToAllVerify1.ini"
    text = src.read_text()
    out = cs.parse_config(src)["output_file"]
    ini = tmp_path / "run.ini"
    ini.write_text(text.replace(out, (tmp_path / "o2a.out").as_posix()))
    r = cs.circuitscape_ini(ini, _solver=O.multi_advanced)
    assert r.maps == {} and (tmp_path / "o2a.out").exists()
    cum, _ = cs.read_raster(tmp_path / "o2a_cum_curmap.asc")
    np.testing.assert_array_equal(cum, r.cum_current)
    want = {p.stem for p in tmp_path.glob("o2a_*map_*.asc")}
    z = np.load(CS / "modes.npz")
    theirs = {"o2a_" + k.split("/")[1][:-4] for k in z.files if k.startswith("oneToAllVerify1/")
              and k.split("/")[1].startswith(("curmap_", "voltmap_"))}
    assert want == theirs
