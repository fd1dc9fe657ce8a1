"""Streaming with resume: the targets solved in consecutive ranges, each call continuing the previous one's maps
(lsb_omni_params.accumulate / target_begin / target_end), give bitwise the maps of one call; a checkpoint after
every range lets an interrupted run resume."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lsb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import landschaft_b200
    return landschaft_b200


def _case(seed=5, shape=(90, 110)):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.normal(0, 1, shape))
    r[rng.random(shape) < 0.03] = np.nan
    return r


KW = dict(block_size=3, buffer=1, flow_potential=True, normalized_current=True, mask_nodata=True)
MAPS = ("cum_currmap", "flow_potential", "normalized_cum_currmap")


def test_ranges_give_the_bits_of_one_call(lsb):
    r = _case()
    one = lsb.omniscape(r, 7, **KW)
    for chunk in (1, 97, 400, 10 ** 6):
        ds = lsb.omniscape(r, 7, chunk_windows=chunk, **KW)
        assert ds.attrs["n_targets"] == one.attrs["n_targets"]
        for k in MAPS:
            np.testing.assert_array_equal(ds[k].values, one[k].values, err_msg=f"{k} chunk {chunk}")


def test_resume_after_an_interruption(lsb, tmp_path):
    from landschaft_b200 import omni
    r = _case(6)
    s = np.where(np.isnan(r), 0.0, 1.0 / np.nan_to_num(r, nan=1.0))
    rt, st = torch.from_numpy(r).cuda(), torch.from_numpy(s).cuda()
    p = omni.make_params(6, 0, 3, flow_potential=True, mask_nodata=True)
    want, _ = omni.run_device(rt, st, p, normalized=True)
    ck = tmp_path / "run.npz"
    part, stats = omni.run_device_streamed(rt, st, p, chunk_windows=150, checkpoint=ck, normalized=True, max_chunks=2)
    assert stats is None and ck.exists() and not bool(np.load(ck)["done"])
    got, stats = omni.run_device_streamed(rt, st, p, chunk_windows=150, checkpoint=ck, normalized=True)
    assert bool(np.load(ck)["done"]) and stats.n_failed == 0
    for k in ("current", "flow_potential", "normalized"):
        assert torch.equal(torch.nan_to_num(got[k], nan=-1.0), torch.nan_to_num(want[k], nan=-1.0)), k
    again, _ = omni.run_device_streamed(rt, st, p, chunk_windows=150, checkpoint=ck, normalized=True)
    assert torch.equal(torch.nan_to_num(again["current"], nan=-1.0), torch.nan_to_num(want["current"], nan=-1.0))
    other = torch.from_numpy(_case(7)).cuda()
    with pytest.raises(ValueError, match="another run"):
        omni.run_device_streamed(other, st, p, chunk_windows=150, checkpoint=ck)
