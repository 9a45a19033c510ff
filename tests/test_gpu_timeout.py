"""The bounded device waits end with WG_E_TIMEOUT instead of hanging, and the
context stays usable afterwards.

The filter's decoupled look-back waits on the status word of the preceding
tile. WG_FILTER_SPIN_LIMIT=0 gives those waits no polls at all, so every tile
after the first gives up at once and publishes its partial prefix: no wait
runs long, every write stays in bounds, and the call must come back with
WG_E_TIMEOUT (the Go wrapper's context-deadline error). The next call with
the normal limit must return the oracle's selection again.
"""
import numpy as np
import pytest

from oracle import binding as ob

pytestmark = pytest.mark.gpu

N = 1 << 22  # 1024 filter tiles of int32


def _data():
    rng = np.random.default_rng(7)
    return rng.integers(0, 1000, N).astype(np.int32)


def test_filter_timeout_is_reported_and_context_recovers(ctx, monkeypatch):
    import wadjet_b200 as wg
    col = _data()
    want = ob.filter_(wg.TYPE_INT32, col, None, wg.OP_LT, 300)
    f = wg.KernelFilter(ctx, 0, wg.OP_LT, 300)
    monkeypatch.setenv("WG_FILTER_SPIN_LIMIT", "0")
    with pytest.raises(wg.WadjetGPUError) as ei:
        f.execute(wg.Batch([wg.Column(wg.TYPE_INT32, col)]))
    assert ei.value.status == wg._abi.WG_E_TIMEOUT
    monkeypatch.delenv("WG_FILTER_SPIN_LIMIT")
    got = f.execute(wg.Batch([wg.Column(wg.TYPE_INT32, col)]))
    np.testing.assert_array_equal(got, want)
    f.close()


def test_filter_timeout_device_entry_points(ctx, monkeypatch):
    import ctypes as C
    import torch
    import wadjet_b200 as wg
    col = _data()
    want = ob.filter_(wg.TYPE_INT32, col, None, wg.OP_LT, 300)
    data = torch.from_numpy(col).cuda()
    out = torch.empty(N, dtype=torch.int32, device="cuda")
    f = wg.KernelFilter(ctx, 0, wg.OP_LT, 300)
    monkeypatch.setenv("WG_FILTER_SPIN_LIMIT", "0")
    with pytest.raises(wg.WadjetGPUError) as ei:
        f.execute_device(wg.Batch([wg.Column(wg.TYPE_INT32, data)]), out)
    assert ei.value.status == wg._abi.WG_E_TIMEOUT
    monkeypatch.delenv("WG_FILTER_SPIN_LIMIT")
    n = f.execute_device(wg.Batch([wg.Column(wg.TYPE_INT32, data)]), out)
    np.testing.assert_array_equal(out[:n].cpu().numpy().view(np.uint32), want)
    f.close()
    # the pipeline still runs on the same context after the expired waits
    agg = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_COUNT, -1)], ndv_hint=1000)
    wg.run_pipeline(ctx, wg.Batch([wg.Column(wg.TYPE_INT32, data)]), agg, filters=[(0, wg.OP_LT, 300)], device=True)
    assert agg.finalize() == 300
    agg.close()
