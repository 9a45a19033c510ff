"""The allocation-free filter entry point, for callers that cannot call cudaMalloc
(a Go operator whose device memory is pre-reserved from the engine's budget, a
thread working beside a global-mode graph capture, a latency-critical serving
thread). It is called through the C ABI and checked against the regular entry
point, wg_filter_execute_device, on two calls in a row: the second call must
not see the first call's leftovers in the shared static scratch. This file is
collected last so a failure here never hides another test's result; it also
passes when run alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(wg, stream, col_t, data, valid, sel, op, value):
    import torch
    kind, i, f = (1, 0, float(value)) if isinstance(value, float) else (0, int(value), 0.0)
    col = wg._abi.wg_column(col_t, 0, data.data_ptr(), valid.data_ptr() if valid is not None else None,
                            int(data.shape[0]))
    n_items = int(sel.shape[0]) if sel is not None else int(data.shape[0])
    out = torch.full((max(1, n_items),), -1, dtype=torch.int32, device=data.device)
    n = C.c_int64(-1)
    st = wg.lib.wg_filter_execute_device_noalloc(stream, C.byref(col), sel.data_ptr() if sel is not None else None,
                                                 n_items, op, kind, i, f, out.data_ptr(), C.byref(n))
    assert st == 0, wg.lib.wg_last_error()
    return out[: n.value].cpu().numpy().view(np.uint32)


def _regular(wg, ctx, col_t, data, valid, sel, op, value):
    import torch
    n_items = int(sel.shape[0]) if sel is not None else int(data.shape[0])
    out = torch.empty(max(1, n_items), dtype=torch.int32, device=data.device)
    f = wg.KernelFilter(ctx, 0, op, value)
    n = f.execute_device(wg.Batch([wg.Column(col_t, data, valid)], sel=sel), out)
    f.close()
    return out[:n].cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("col_t,dtype,value", [(1, np.int32, 500), (2, np.int64, 500), (4, np.float64, 0.5)])
def test_noalloc_matches_regular_entry_point_twice(ctx, col_t, dtype, value):
    import torch
    import wadjet_b200 as wg
    rng = np.random.default_rng(col_t)
    stream = ctx.stream
    results = []
    # two calls in a row on different inputs: a large one, then a smaller one whose
    # tiles reuse the status words the first call left behind
    for n, use_nulls, use_sel in ((3_000_017, True, False), (1_000_003, False, True)):
        host = (rng.random(n) if dtype == np.float64 else rng.integers(0, 1000, n)).astype(dtype)
        data = torch.from_numpy(host).cuda()
        valid = None
        if use_nulls:
            valid = torch.from_numpy(wg.pack_validity(rng.random(n) > 0.1).view(np.int64)).cuda()
        sel = torch.from_numpy(np.sort(rng.choice(n, n // 3, replace=False)).astype(np.int32)).cuda() if use_sel \
            else None
        want = _regular(wg, ctx, col_t, data, valid, sel, wg.OP_LT, value)
        got = _noalloc(wg, stream, col_t, data, valid, sel, wg.OP_LT, value)
        np.testing.assert_array_equal(got, want)
        results.append(len(got))
    assert all(r > 0 for r in results)


def test_noalloc_rejects_inputs_over_the_limit(ctx):
    import wadjet_b200 as wg
    import torch
    data = torch.zeros(16, dtype=torch.int32, device="cuda")
    col = wg._abi.wg_column(1, 0, data.data_ptr(), None, 16)
    n = C.c_int64(-1)
    over = wg._abi.WG_E_INVALID
    st = wg.lib.wg_filter_execute_device_noalloc(ctx.stream, C.byref(col), None, (1 << 26) + 1, wg.OP_EQ, 0, 0, 0.0,
                                                 data.data_ptr(), C.byref(n))
    assert st == over
    assert b"limit" in wg.lib.wg_last_error()


def test_noalloc_rejects_more_items_than_the_column_holds(ctx):
    # without a selection vector the items are the column's rows; a larger count
    # would read past the column, so the call refuses it before any launch
    import wadjet_b200 as wg
    import torch
    data = torch.zeros(1000, dtype=torch.int32, device="cuda")
    out = torch.empty(2000, dtype=torch.int32, device="cuda")
    col = wg._abi.wg_column(1, 0, data.data_ptr(), None, 1000)
    n = C.c_int64(-1)
    st = wg.lib.wg_filter_execute_device_noalloc(ctx.stream, C.byref(col), None, 1001, wg.OP_EQ, 0, 0, 0.0,
                                                 out.data_ptr(), C.byref(n))
    assert st == wg._abi.WG_E_INVALID
    assert b"column length" in wg.lib.wg_last_error()


def test_noalloc_timeout_then_clean_call(ctx, monkeypatch):
    # an expired look-back wait leaves its mark in the shared scratch's error word;
    # the next call must clear it and return the regular entry point's selection
    import torch
    import wadjet_b200 as wg
    rng = np.random.default_rng(11)
    host = rng.integers(0, 1000, 1 << 22).astype(np.int32)
    data = torch.from_numpy(host).cuda()
    monkeypatch.setenv("WG_FILTER_SPIN_LIMIT", "0")
    kind_i = int(500)
    col = wg._abi.wg_column(1, 0, data.data_ptr(), None, int(data.shape[0]))
    out = torch.empty(int(data.shape[0]), dtype=torch.int32, device="cuda")
    n = C.c_int64(-1)
    st = wg.lib.wg_filter_execute_device_noalloc(ctx.stream, C.byref(col), None, int(data.shape[0]), wg.OP_LT, 0,
                                                 kind_i, 0.0, out.data_ptr(), C.byref(n))
    assert st == wg._abi.WG_E_TIMEOUT
    monkeypatch.delenv("WG_FILTER_SPIN_LIMIT")
    want = _regular(wg, ctx, 1, data, None, None, wg.OP_LT, 500)
    got = _noalloc(wg, ctx.stream, 1, data, None, None, wg.OP_LT, 500)
    np.testing.assert_array_equal(got, want)
