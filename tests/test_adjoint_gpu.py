"""The adjoint of the cumulative current on the GPU.

* against the FP64 adjoint of the oracle (``orc_omniscape_grad``, which uses the oracle's direct solve):
  J to 1e-9 and every gradient entry to 1e-6 of the gradient's largest magnitude, FP64 and FP32+refinement;
* against central finite differences of the GPU's own FP64 forward, on a small map and on the 512 x 512,
  radius-24 workload with J = sum of the current over rows and columns 224-287 at 200 random cells: at step
  1e-3 relative, at most 1e-4 relative error at 90% of the cells or more; at the others (a slope jump of J
  lies within the step) at step 1e-4 or 1e-5 relative;
* through ``torch.autograd``: the backward of ``omniscape_current`` is the same vector-Jacobian product.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lsb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import landschaft_b200
    return landschaft_b200


def _case(seed, shape, nodata=0.04):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.normal(0, 0.7, shape))
    r[rng.random(shape) < nodata] = np.nan
    s = np.where(rng.random(shape) < 0.5, rng.uniform(0.5, 1.5, shape), 0.0)
    w = np.zeros(shape)
    w[shape[0] // 3: 2 * shape[0] // 3, shape[1] // 4: 3 * shape[1] // 4] = 1.0
    w += 0.1 * rng.random(shape)
    return r, s, w


def _grad(lsb, r, s, w, radius, **kw):
    from landschaft_b200 import omni
    p = omni.make_params(radius, correct_artifacts=False, use_graph=False, **kw)
    t = [torch.from_numpy(x).cuda() for x in (r, s, w)]
    J, gr, gs, stats = lsb.grad_device(*t, p)
    assert stats.n_failed == 0
    return float(J.item()), gr.cpu().numpy(), gs.cpu().numpy()


CASES = [dict(radius=4), dict(radius=6, buffer=1, four_neighbors=True), dict(radius=5, block_size=3),
         dict(radius=4, edge_weights="series"), dict(radius=5, resistance_is_conductance=True)]


@pytest.mark.parametrize("solver", ["fp64", "fp32-refine"])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_adjoint_matches_the_oracle(lsb, case, solver):
    kw = dict(CASES[case])
    r, s, w = _case(40 + case, (31, 36))
    radius = kw.pop("radius")
    series = kw.get("edge_weights") == "series"
    J, gr, gs = _grad(lsb, r, s, w, radius, solver=solver, **kw)
    Jo, gro, gso = oracle.omniscape_grad(r, s, w, radius, buffer=kw.get("buffer", 0),
                                         block_size=kw.get("block_size", 1), four=kw.get("four_neighbors", False),
                                         ric=kw.get("resistance_is_conductance", False), series=series)
    assert abs(J - Jo) <= 1e-9 * abs(Jo)
    for got, want in ((gr, gro), (gs, gso)):
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 * np.abs(want).max())


STEPS = (1e-3, 1e-4, 1e-5)


def _fd_errors(J, r0, adj):
    """Relative error of the adjoint against central differences of J at each relative step of STEPS.

    J (as a function of the perturbation of one cell) is piecewise smooth: the node current sums the positive
    branch currents, so its slope jumps wherever a branch current in any window changes sign.  A step that spans
    such a point gives a central difference that is no derivative; the smaller steps then still see one smooth
    piece (and a too-small step drowns in the solver's rounding, so no single step serves every cell).
    """
    errs = []
    for h_rel in STEPS:
        h = h_rel * r0
        fd = (J(h) - J(-h)) / (2 * h)
        errs.append(abs(fd - adj) / max(abs(fd), 1e-300))
    return errs


def _fd_verdict(errs, grads, gmax, min_first=0.9):
    errs = np.array(errs)
    big = np.abs(np.array(grads)) > 1e-6 * gmax
    assert big.sum() >= 10
    first = errs[big, 0] <= 1e-4
    # at most a tenth of the cells have a slope jump within 1e-3 relative of their value, and at every
    # cell one of the steps agrees with the adjoint to 1e-4
    assert first.mean() >= min_first, (first.mean(), errs[big][~first])
    assert np.all(errs[big].min(axis=1) <= 1e-4), errs[big][errs[big].min(axis=1) > 1e-4]


def test_adjoint_matches_finite_differences_small(lsb):
    from landschaft_b200 import omni
    r, s, w = _case(7, (40, 44))
    rng = np.random.default_rng(1)
    cells = [(y, x) for y, x in zip(rng.integers(0, 40, 30), rng.integers(0, 44, 30)) if not np.isnan(r[y, x])]
    _, gr, _ = _grad(lsb, r, s, w, 6, solver="fp32-refine")
    p = omni.make_params(6, correct_artifacts=False, solver="fp64", use_graph=False)
    wt, st = torch.from_numpy(w).cuda(), torch.from_numpy(s).cuda()
    errs = []
    for y, x in cells:
        def J(d):
            rr = r.copy()
            rr[y, x] += d
            out, _ = omni.run_device(torch.from_numpy(rr).cuda(), st, p)
            return float((torch.nan_to_num(out["current"]) * wt).sum().item())
        errs.append(_fd_errors(J, r[y, x], gr[y, x]))
    _fd_verdict(errs, [gr[c] for c in cells], np.abs(gr).max(), min_first=0.75)


def test_adjoint_config_512_finite_differences(lsb):
    # the 512 x 512, radius 24 workload (sources 1 / resistance, held fixed): J = sum of the cumulative current
    # over rows and columns 224-287; 200 random cells within 2 radii of the patch (farther cells have no
    # gradient).  Differences are taken on a crop of +-2 radii around the cell: every window that contains the
    # cell lies in the crop with the same clipping, and windows that do not contain it cancel in the difference.
    from landschaft_b200 import omni, synthetic
    r, s, w, kw = synthetic.adjoint_512()
    D = kw["radius"]
    _, gr, _ = _grad(lsb, r, s, w, D, solver="fp32-refine")
    p64 = omni.make_params(D, correct_artifacts=False, solver="fp64", use_graph=False)
    rng = np.random.default_rng(0)
    cells = []
    while len(cells) < 200:
        y, x = (int(v) for v in rng.integers(224 - 2 * D, 288 + 2 * D, 2))
        if not np.isnan(r[y, x]):
            cells.append((y, x))
    errs = []
    for y, x in cells:
        y0, y1 = max(y - 2 * D, 0), min(y + 2 * D + 1, 512)
        x0, x1 = max(x - 2 * D, 0), min(x + 2 * D + 1, 512)
        rc = np.ascontiguousarray(r[y0:y1, x0:x1])
        sc = torch.from_numpy(np.ascontiguousarray(s[y0:y1, x0:x1])).cuda()
        wc = torch.from_numpy(np.ascontiguousarray(w[y0:y1, x0:x1])).cuda()

        def J(d):
            rr = rc.copy()
            rr[y - y0, x - x0] += d
            out, _ = omni.run_device(torch.from_numpy(rr).cuda(), sc, p64)
            return float((torch.nan_to_num(out["current"]) * wc).sum().item())
        errs.append(_fd_errors(J, r[y, x], gr[y, x]))
    _fd_verdict(errs, [gr[c] for c in cells], np.abs(gr).max())


def test_autograd_is_the_vector_jacobian_product(lsb):
    r, s, w = _case(9, (28, 30))
    rt = torch.from_numpy(r).cuda().requires_grad_(True)
    st = torch.from_numpy(s).cuda().requires_grad_(True)
    cur = lsb.omniscape_current(rt, st, 5)
    wt = torch.from_numpy(w).cuda()
    (torch.nan_to_num(cur) * wt).sum().backward()
    J, gr, gs = _grad(lsb, r, s, w, 5)
    np.testing.assert_allclose(rt.grad.cpu().numpy(), gr, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(st.grad.cpu().numpy(), gs, rtol=1e-12, atol=1e-300)
