"""The autotuner on the GPU: it times every candidate on a sample, installs the fastest, and calls on "auto" then
run exactly the chosen configuration (bitwise the same maps as the explicit call)."""

from __future__ import annotations

import ctypes as C

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lsb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import landschaft_b200
    yield landschaft_b200
    landschaft_b200.clear_tuning()


def test_autotune_installs_the_fastest_candidate(lsb):
    from landschaft_b200 import _native as N
    from landschaft_b200 import omni, synthetic
    r, s, kw = synthetic.omni_128(0)
    lsb.clear_tuning()
    entry = lsb.autotune(r, s, kw["radius"], block_size=1, windows=400)
    times = {k: v for k, v in entry["window_ms"].items() if v is not None}
    assert set(entry["window_ms"]) == {"mg/512", "mg/256", "mg/128", "jacobi/512", "jacobi/256", "jacobi/128"}
    best = f'{entry["preconditioner"]}/{entry["threads_per_window"]}'
    assert times[best] == min(times.values())
    pc, nt = C.c_int32(), C.c_int32()
    assert N.load().lsb_tune_get(17, 0, 0, N.PREC_FP32_REFINE, C.byref(pc), C.byref(nt)) == 1
    assert (pc.value, nt.value) == (omni.PRECONDITIONERS.index(entry["preconditioner"]), entry["threads_per_window"])
    rt, st = torch.from_numpy(r).cuda(), torch.from_numpy(s).cuda()
    auto, sa = omni.run_device(rt, st, omni.make_params(8))
    expl, _ = omni.run_device(rt, st, omni.make_params(8, preconditioner=entry["preconditioner"],
                                                       threads_per_window=entry["threads_per_window"]))
    assert sa.threads_per_window == entry["threads_per_window"] and sa.preconditioner == pc.value
    assert torch.equal(auto["current"], expl["current"])
    lsb.clear_tuning()
    # the built-in rule again (a new table generation: the graph cached for the tuned call is not replayed)
    _, sd = omni.run_device(rt, st, omni.make_params(8))
    assert sd.preconditioner == omni.PRECONDITIONERS.index("mg") and sd.threads_per_window == 256
