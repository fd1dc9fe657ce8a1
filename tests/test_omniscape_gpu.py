"""Parity of the GPU path (through the C ABI) with the oracle and the reference's golden vectors.

Tolerances:
* golden cases: the reference's own test bar (tests/test_omniscape.py:150-157 of the reference): identical NaN
  and zero patterns, rtol 1e-9 and atol 1e-13 x max against Omniscape.jl + CHOLMOD, for both solvers;
* against the oracle: identical NaN and zero patterns, rtol 1e-9 / atol 1e-12 x max, and for the cumulative
  current the north-star metric max |gpu - oracle| / |oracle| <= 1e-6 over cells with |oracle| > 1e-12 x max;
* bitwise: determinism run to run, graph replay vs direct launches, batching.
"""

from __future__ import annotations

import ctypes as C
import warnings

import numpy as np
import pytest

import oracle
from tests.test_oracle import GOLD, OUTPUTS, check_golden, golden_cases, golden_kwargs

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SOLVERS = ("fp64", "fp32-refine")


@pytest.fixture(scope="module")
def lsb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import landschaft_b200
    from landschaft_b200 import _native
    _native.load()
    return landschaft_b200


def _map(seed=1, shape=(40, 50), nodata=0.05):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.normal(0.5, 1.0, shape))
    r[rng.random(shape) < nodata] = np.nan
    return r


def max_rel(ours, want):
    top = np.nanmax(np.abs(want))
    m = ~np.isnan(want) & (np.abs(want) > 1e-12 * top)
    if not m.any():
        return 0.0
    return float(np.max(np.abs(ours[m] - want[m]) / np.abs(want[m])))


def _values(ds, k):
    v = ds[k]
    return np.asarray(v.values if hasattr(v, "values") else v)


def check_against(ds, ref, rtol=1e-9, metric=1e-6):
    for k in OUTPUTS:
        if k not in ref:
            assert k not in ds
            continue
        ours, want = _values(ds, k), ref[k]
        np.testing.assert_array_equal(np.isnan(ours), np.isnan(want), err_msg=k)
        np.testing.assert_array_equal(ours == 0, want == 0, err_msg=k)
        top = np.nanmax(np.abs(want)) if np.isfinite(want).any() else 1.0
        np.testing.assert_allclose(ours, want, rtol=rtol, atol=1e-12 * top, err_msg=k)
        if k == "cum_currmap":
            assert max_rel(ours, want) <= metric


@pytest.mark.parametrize("solver", SOLVERS)
@pytest.mark.parametrize("name", golden_cases())
def test_matches_omniscape_golden(lsb, name, solver):
    z = np.load(GOLD / "omniscape_golden.npz")
    kw, source = golden_kwargs(z, name)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ds = lsb.omniscape(z[f"{name}/resistance"], source=source, solver=solver, **kw)
    check_golden({k: ds[k].values for k in ds.data_vars}, z, name)


CASES = [
    dict(radius=5, block_size=1),
    dict(radius=6, block_size=3, buffer=2, flow_potential=True, normalized_current=True),
    dict(radius=4, block_size=5, buffer=1, four_neighbors=True, flow_potential=True),
    dict(radius=7, block_size=3, correct_artifacts=False, resistance_is_conductance=True),
    dict(radius=3, block_size=7, buffer=4, normalized_current=True),
    dict(radius=9, block_size=1, four_neighbors=True, mask_nodata=False),
    dict(radius=6, block_size=3, edge_weights="series", flow_potential=True),
    dict(radius=12, block_size=5, buffer=3, flow_potential=True, normalized_current=True),
    dict(radius=5, block_size=3, precision="single", flow_potential=True),
    dict(radius=2, block_size=1, r_cutoff=3.0),
]


@pytest.mark.parametrize("solver", SOLVERS)
@pytest.mark.parametrize("case", range(len(CASES)))
def test_matches_oracle(lsb, case, solver):
    kw = dict(CASES[case])
    r = _map(20 + case, (43, 51))
    if kw.get("resistance_is_conductance"):
        r = 1 / r
    series = kw.pop("edge_weights", "average") == "series"
    ds = lsb.omniscape(r, solver=solver, edge_weights="series" if series else "average", **kw)
    ref = oracle.omniscape(r, series=series, **kw)
    if kw.get("precision") == "single":
        for k in ref:
            if k != "attrs":
                assert ds[k].values.dtype == np.float32
        ref = {k: v.astype(np.float64) for k, v in ref.items() if k != "attrs"}
        ds = {k: ds[k].values.astype(np.float64) for k in ds.data_vars}
        check_against(ds, ref, rtol=1e-6)
        return
    ref.pop("attrs")
    check_against(ds, ref)


def test_conditions(lsb):
    rng = np.random.default_rng(4)
    r = _map(4, (33, 41))
    c1 = rng.uniform(0, 10, r.shape)
    c1f = c1 + rng.normal(0, 1, r.shape)
    c2 = rng.integers(0, 3, r.shape).astype(float)
    c2[rng.random(r.shape) < 0.1] = np.nan
    for kw in (dict(condition1=c1, condition1_lower=-2.0, condition1_upper=1.5),
               dict(condition1=c1, condition1_future=c1f, compare_to_future="1", condition1_lower=-2.0,
                    condition1_upper=1.5, condition2=c2, comparison2="equal"),
               dict(condition1=c2, comparison1="equal", block_size=5)):
        kw = dict(kw)
        bs = kw.pop("block_size", 3)
        ds = lsb.omniscape(r, 5, block_size=bs, **kw)
        ref = oracle.omniscape(r, 5, block_size=bs, **kw)
        ref.pop("attrs")
        check_against(ds, ref)


def test_condition_all_nodata_raises(lsb):
    r = _map(5, (20, 20))
    c = np.full(r.shape, np.nan)
    with pytest.raises(RuntimeError, match="condition"):
        lsb.omniscape(r, 3, condition1=c)


def test_config_128_full(lsb):
    # the 128 x 128, radius 8 workload, every window, against the oracle
    from landschaft_b200 import synthetic
    r, s, kw = synthetic.omni_128()
    ref = oracle.omniscape(r, kw["radius"], source=s, flow_potential=True, normalized_current=True)
    ref.pop("attrs")
    for solver in SOLVERS:
        ds = lsb.omniscape(r, kw["radius"], source=s, flow_potential=True, normalized_current=True, solver=solver)
        assert ds.attrs["n_targets"] == 128 * 128
        check_against(ds, ref)


def test_config_4096_radius64_crop(lsb):
    # the 4096 x 4096, radius 64, block 5 workload (129-cell windows, solver arrays in global scratch): a
    # 256 x 256 crop, every window, against the reference's own driver, at the 1e-6 bar of the FP32 solve
    from landschaft_b200 import synthetic
    r, s, kw = synthetic.omni_4096()
    r = np.ascontiguousarray(r[3500:3756, 3000:3256])
    s = np.ascontiguousarray(s[3500:3756, 3000:3256])
    impl = "ref" if oracle.REF_AVAILABLE else "port"
    ref = oracle.core_omniscape(r, s, kw["radius"], 0, kw["block_size"], False, False, True, False, impl=impl)
    ds, stats = lsb.omniscape(r, kw["radius"], source=s, block_size=kw["block_size"], mask_nodata=False,
                              return_stats=True)
    assert ds.attrs["n_targets"] == ref["n_targets"] >= 500
    assert stats["n_failed"] == 0
    cur = _values(ds, "cum_currmap")
    assert max_rel(cur, ref["current"]) <= 1e-6
    np.testing.assert_array_equal(cur == 0, ref["current"] == 0)


def test_deterministic_and_graph_replay(lsb):
    r = _map(3, (50, 60))
    s = np.where(np.isnan(r), 0, 1 / np.nan_to_num(r, nan=1))
    kw = dict(source=s, block_size=3, buffer=2, flow_potential=True, normalized_current=True)
    a = lsb.omniscape(r, 6, **kw)
    b = lsb.omniscape(r, 6, **kw)
    for k in OUTPUTS:
        np.testing.assert_array_equal(a[k].values, b[k].values)
    # graph replay and direct launches give the same bits
    from landschaft_b200 import omni as om
    rt = torch.from_numpy(r).cuda()
    st = torch.from_numpy(s).cuda()
    outs = []
    for use_graph in (True, True, False):
        p = om.make_params(6, 2, 3, flow_potential=True, use_graph=use_graph)
        out, stats = om.run_device(rt, st, p)
        outs.append({k: v.clone() for k, v in out.items()})
    for o in outs[1:]:
        for k in outs[0]:
            assert torch.equal(o[k], outs[0][k])


def test_batches_give_the_same_bits(lsb):
    r = _map(6, (45, 47))
    a = lsb.omniscape(r, 5, block_size=3, flow_potential=True)
    w = 2 * 5 + 1
    b, st = lsb.omniscape(r, 5, block_size=3, flow_potential=True, memory_limit=7 * w * w * 16, return_stats=True)
    assert st["batches"] > 3
    np.testing.assert_array_equal(a.cum_currmap.values, b.cum_currmap.values)
    np.testing.assert_array_equal(a.flow_potential.values, b.flow_potential.values)


def test_options_and_masks(lsb):
    # tests/test_omniscape.py:60-78 of the reference
    r = _map(4)
    with pytest.warns(UserWarning, match="block_size is even"):
        ds = lsb.omniscape(r, 5, block_size=2, flow_potential=True, normalized_current=True)
    assert ds.attrs["block_size"] == 3
    nodata = np.isnan(r)
    for k in OUTPUTS:
        assert np.isnan(ds[k].values[nodata]).all() and not np.isnan(ds[k].values[~nodata]).any()
    ds2 = lsb.omniscape(r, 5, block_size=3, flow_potential=True, normalized_current=True, mask_nodata=False)
    assert not np.isnan(ds2.cum_currmap.values).any()
    np.testing.assert_array_equal(ds2.cum_currmap.values[~nodata], ds.cum_currmap.values[~nodata])
    fp = ds2.flow_potential.values
    with np.errstate(invalid="ignore", divide="ignore"):
        expect = np.where((ds2.cum_currmap.values == 0) & (fp == 0), 0, ds2.cum_currmap.values / fp)
    np.testing.assert_array_equal(ds2.normalized_cum_currmap.values, expect)
    assert list(lsb.omniscape(r, 5).data_vars) == ["cum_currmap"]
    assert list(lsb.omniscape(r, 5, normalized_current=True).data_vars) == ["cum_currmap", "normalized_cum_currmap"]


def test_source_from_resistance_and_threshold(lsb):
    # tests/test_omniscape.py:81-100 of the reference
    r = _map(5)
    expect = np.where(np.isnan(r) | (1 / r < 0.5), 0, 1 / r)
    a = lsb.omniscape(r, 4, r_cutoff=2.0)
    b = lsb.omniscape(r, 4, source=expect)
    np.testing.assert_array_equal(a.cum_currmap.values, b.cum_currmap.values)
    c = lsb.omniscape(1 / r, 4, source=expect, resistance_is_conductance=True)
    np.testing.assert_allclose(c.cum_currmap.values, a.cum_currmap.values, rtol=1e-10)
    r = _map(6)
    s = np.random.default_rng(6).uniform(0, 1, r.shape)
    s[::7, ::5] = np.nan
    a = lsb.omniscape(r, 4, source=s, source_threshold=0.4)
    b = lsb.omniscape(r, 4, source=np.where(np.isnan(s) | (s < 0.4), 0, s))
    np.testing.assert_array_equal(a.cum_currmap.values, b.cum_currmap.values)


def test_single_target_is_one_advanced_solve(lsb):
    r = _map(2, (15, 15))
    r[np.isnan(r)] = 1.0
    s = np.zeros(r.shape)
    s[7, 7] = 1.0
    s[5, 9] = 2.0
    ds = lsb.omniscape(r, 4, source=s)
    assert ds.attrs["n_targets"] == 2
    total = np.zeros(r.shape)
    for (ty, tx), amps, other in [((7, 7), 1.0, (5, 9)), ((5, 9), 2.0, (7, 7))]:
        yy, xx = np.mgrid[:15, :15]
        g = np.where((yy - ty) ** 2 + (xx - tx) ** 2 <= 16, 1 / r, 0.0)
        src = np.zeros(r.shape)
        src[other] = amps
        gr = np.zeros(r.shape)
        gr[ty, tx] = np.inf
        total += oracle.advanced(g, src, gr)[0]
    np.testing.assert_allclose(ds.cum_currmap.values, total, rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("args", [(4, 1, 1, False), (6, 2, 5, False), (5, 0, 3, True), (8, 3, 7, False)])
def test_correction_factors(lsb, args):
    c = lsb.omniscape_correction(*args, 50, 50)
    want = oracle.correction(*args, 50, 50)
    assert c.shape == want.shape
    np.testing.assert_allclose(c, want, rtol=1e-9)
    if args[2] == 1:
        np.testing.assert_array_equal(c, 1.0)


@pytest.mark.parametrize("shape,radius,bs", [((1, 1), 3, 1), ((1, 7), 2, 1), ((7, 1), 2, 1), ((5, 5), 10, 1),
                                             ((9, 9), 0, 1), ((4, 4), 2, 5), ((3, 40), 6, 3)])
def test_edge_shapes(lsb, shape, radius, bs):
    r = _map(30, shape, nodata=0.0)
    ds = lsb.omniscape(r, radius, block_size=bs, flow_potential=True, normalized_current=True)
    ref = oracle.omniscape(r, radius, block_size=bs, flow_potential=True, normalized_current=True)
    ref.pop("attrs")
    check_against(ds, ref)


def test_no_targets_and_all_nodata(lsb):
    r = _map(7, (20, 20))
    ds = lsb.omniscape(r, 3, source=np.zeros(r.shape), flow_potential=True)
    assert ds.attrs["n_targets"] == 0
    assert np.nansum(ds.cum_currmap.values) == 0 and np.nansum(ds.flow_potential.values) == 0
    ds = lsb.omniscape(np.full((10, 12), np.nan), 3, source=np.ones((10, 12)))
    assert np.isnan(ds.cum_currmap.values).all()


def test_c_abi_direct(lsb):
    # the C entry point with raw device pointers, as a non-Python host would call it
    from landschaft_b200 import _native as N
    lib = N.load()
    r = _map(11, (30, 31))
    s = np.where(np.isnan(r), 0.0, 1 / np.nan_to_num(r, nan=1.0))
    rt, st = torch.from_numpy(r).cuda(), torch.from_numpy(s).cuda()
    cur = torch.empty_like(rt)
    p = N.default_params()
    p.radius, p.block_size = 4, 3
    p.mask_nodata = 1
    need = C.c_size_t(0)
    assert lib.lsb_omniscape_workspace_size(31, 30, C.byref(p), C.byref(need)) == 0
    ws = torch.empty(need.value, dtype=torch.uint8, device="cuda")
    err = C.create_string_buffer(256)
    stats = N.Stats()
    stream = torch.cuda.Stream()
    rc = lib.lsb_omniscape(rt.data_ptr(), st.data_ptr(), 31, 30, C.byref(p), cur.data_ptr(), None, None,
                           ws.data_ptr(), need.value, C.byref(stats), err, 256, stream.cuda_stream)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    want = oracle.omniscape(r, 4, block_size=3)["cum_currmap"]
    got = cur.cpu().numpy()
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-13 * np.nanmax(want))
    assert stats.n_targets > 0 and stats.n_failed == 0 and lib.lsb_last_launch_count() > 0
    # errors come back as codes with a message, not exceptions
    p.block_size = 2
    assert lib.lsb_omniscape_workspace_size(31, 30, C.byref(p), C.byref(need)) == N.LSB_ERR_ARGUMENT
    rc = lib.lsb_omniscape(rt.data_ptr(), st.data_ptr(), 31, 30, C.byref(p), cur.data_ptr(), None, None,
                           ws.data_ptr(), 16, None, err, 256, None)
    assert rc == N.LSB_ERR_ARGUMENT and b"odd" in err.value
    p.block_size = 3
    rc = lib.lsb_omniscape(rt.data_ptr(), st.data_ptr(), 31, 30, C.byref(p), cur.data_ptr(), None, None,
                           ws.data_ptr(), 16, None, err, 256, None)
    assert rc == N.LSB_ERR_WORKSPACE
