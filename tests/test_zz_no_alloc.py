"""The entry point without a workspace (``lsb_omniscape_noalloc``), for callers that cannot call cudaMalloc.

Some hosts cannot allocate device memory when they call this library: their device memory is already reserved
by another framework's pool, or they must not pay the implicit device synchronization an allocation can cause.
For them ``lsb_omniscape_noalloc`` runs the same solve out of one static device array that the library holds.
This test calls it through the C ABI, twice in a row (the array keeps the previous call's contents), and checks
both results against ``lsb_omniscape`` with a workspace, at the tolerance of the other GPU tests (rtol 1e-9,
atol 1e-12 of the maximum; identical NaN and zero patterns).  It also checks that a raster too large for the
static array is refused with a message.  The file is named so that pytest collects it last.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _rasters(seed, shape):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.normal(0.5, 1.0, shape))
    r[rng.random(shape) < 0.05] = np.nan
    s = np.where(np.isnan(r), 0.0, 1.0 / np.nan_to_num(r, nan=1.0))
    return r, s


def _check(got, want):
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
    np.testing.assert_array_equal(got == 0, want == 0)
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * np.nanmax(np.abs(want)))


def test_noalloc_matches_the_workspace_entry_point_twice():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from landschaft_b200 import _native as N
    lib = N.load()
    ny, nx = 96, 110
    r, s = _rasters(12, (ny, nx))
    rt, st = torch.from_numpy(r).cuda(), torch.from_numpy(s).cuda()
    p = N.default_params()
    p.radius, p.buffer, p.block_size = 29, 1, 3  # windows of 61 x 61: the static path must stream in batches
    p.flow_potential = 1
    p.mask_nodata = 1
    p.use_graph = 0
    err = C.create_string_buffer(512)
    stream = torch.cuda.Stream()
    # the existing entry point, with a caller-allocated workspace
    need = C.c_size_t(0)
    assert lib.lsb_omniscape_workspace_size(nx, ny, C.byref(p), C.byref(need)) == 0
    ws = torch.empty(need.value, dtype=torch.uint8, device="cuda")
    want_c, want_f, want_n = (torch.empty_like(rt) for _ in range(3))
    rc = lib.lsb_omniscape(rt.data_ptr(), st.data_ptr(), nx, ny, C.byref(p), want_c.data_ptr(), want_f.data_ptr(),
                           want_n.data_ptr(), ws.data_ptr(), need.value, C.byref(N.Stats()), err, 512,
                           stream.cuda_stream)
    assert rc == 0, err.value
    stream.synchronize()
    # the same call without a workspace, twice in a row: the static scratch keeps the first call's contents
    for _ in range(2):
        cur, fp, norm = (torch.full_like(rt, -1.0) for _ in range(3))
        stats = N.Stats()
        rc = lib.lsb_omniscape_noalloc(rt.data_ptr(), st.data_ptr(), nx, ny, C.byref(p), cur.data_ptr(),
                                       fp.data_ptr(), norm.data_ptr(), C.byref(stats), err, 512, stream.cuda_stream)
        assert rc == 0, err.value
        stream.synchronize()
        assert stats.n_targets > 0 and stats.n_failed == 0
        _check(cur.cpu().numpy(), want_c.cpu().numpy())
        _check(fp.cpu().numpy(), want_f.cpu().numpy())
        _check(norm.cpu().numpy(), want_n.cpu().numpy())


def test_noalloc_refuses_rasters_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from landschaft_b200 import _native as N
    lib = N.load()
    p = N.default_params()
    p.radius, p.block_size = 4, 1
    err = C.create_string_buffer(512)
    # 6000 x 6000 block centres: the per-target tables alone exceed the static array; refused before any work
    rc = lib.lsb_omniscape_noalloc(None, None, 6000, 6000, C.byref(p), None, None, None, None, err, 512, None)
    assert rc == N.LSB_ERR_WORKSPACE
    assert b"static" in err.value
