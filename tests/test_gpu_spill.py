"""Aggregations whose hash table does not fit the HBM ledger (memory.Tracker's
budget turned into device bytes): the rows are partitioned by key hash into
pinned host memory while they are consumed, and finalize aggregates one
partition at a time in a small table. Results must equal the oracle's, the
ledger's peak must stay within the budget, and a reset aggregate must give the
same answer again."""
import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import DEC_DTYPE, assert_groups_equal

pytestmark = pytest.mark.gpu

I32, I64, F64, DEC = 1, 2, 4, 17
MB = 1 << 20


def to_host_dec(t):
    return t.cpu().numpy().reshape(-1).view(DEC_DTYPE)


def test_spilled_packed_key_aggregate_matches_oracle():
    """GROUP BY (a int32, b int64) over 2^22 rows (~3.9M groups) with a 512 MB budget: the full
    table (just over 512 MB) does not fit; the compact result (~250 MB) and its export do."""
    import wadjet_b200 as wg
    from wadjet_b200 import synth
    budget = 512 * MB
    with wg.Context(0, hbm_budget=budget, pinned_spill=2 << 30) as ctx:
        n = 1 << 22
        a, b, amt, x = synth.highcard(ctx, n)
        aggs = [wg.AggColumn(wg.AGG_SUM, 2), wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_MIN, 3),
                wg.AggColumn(wg.AGG_MAX, 3)]
        g = wg.HashAggregate(ctx, [0, 1], aggs, ndv_hint=1 << 22)
        cuts = [0, 1 << 20, 3 << 20, n]  # three consume calls, three spilled runs
        for lo, hi in zip(cuts[:-1], cuts[1:]):
            wg.run_pipeline(ctx, wg.Batch([wg.Column(I32, a[lo:hi]), wg.Column(I64, b[lo:hi]),
                                           wg.Column(DEC, amt[lo:hi], scale=2), wg.Column(F64, x[lo:hi])]),
                            g, device=True)
        g.finalize()
        first = g.export()
        assert ctx.ledger()["peak"] <= budget
        ha, hb, hamt, hx = a.cpu().numpy(), b.cpu().numpy(), to_host_dec(amt), x.cpu().numpy()
        o = ob.Agg([0, 1], [(0, 2, 0), (1, -1, 0), (2, 3, 0), (3, 3, 0)])
        ob.pipeline(ob.HostBatch([(I32, ha, None, 0), (I64, hb, None, 0), (DEC, hamt, None, 2), (F64, hx, None, 0)]),
                    o, threads=8)
        kinds = ["sum_d", "count", "min_f", "max_f"]
        assert_groups_equal(first, o.export(), kinds)
        # the same aggregate, reset, fed in one call
        g.reset()
        wg.run_pipeline(ctx, wg.Batch([wg.Column(I32, a), wg.Column(I64, b), wg.Column(DEC, amt, scale=2),
                                       wg.Column(F64, x)]), g, device=True)
        g.finalize()
        assert_groups_equal(g.export(), o.export(), kinds)
        g.close()


def test_spilled_int_key_aggregate_with_filter_matches_oracle():
    """WHERE flag < 7 GROUP BY k (int64, ~0.9M groups) over 2^21 rows with an 80 MB budget (the
    full table takes 84 MB); the consume call is cut into several windows, each spilled as its own run."""
    import torch
    import wadjet_b200 as wg
    rng = np.random.default_rng(5)
    n = 1 << 21
    hk = rng.integers(0, 1 << 20, n).astype(np.int64) * 7919 - 12345
    hv = rng.integers(-10**6, 10**6, n).astype(np.int64)
    hf = rng.random(n)
    hflag = rng.integers(0, 10, n).astype(np.int32)
    budget = 80 * MB
    with wg.Context(0, hbm_budget=budget, pinned_spill=1 << 30) as ctx:
        cols = [torch.from_numpy(c).cuda() for c in (hk, hv, hf, hflag)]
        aggs = [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_MIN, 2),
                wg.AggColumn(wg.AGG_MAX, 2)]
        g = wg.HashAggregate(ctx, [0], aggs, ndv_hint=1 << 20)
        wg.run_pipeline(ctx, wg.Batch([wg.Column(I64, cols[0]), wg.Column(I64, cols[1]), wg.Column(F64, cols[2]),
                                       wg.Column(I32, cols[3])]), g, filters=[(3, wg.OP_LT, 7)], device=True)
        g.finalize()
        assert ctx.ledger()["peak"] <= budget
        o = ob.Agg([0], [(0, 1, 0), (1, -1, 0), (2, 2, 0), (3, 2, 0)])
        ob.pipeline(ob.HostBatch([(I64, hk, None, 0), (I64, hv, None, 0), (F64, hf, None, 0), (I32, hflag, None, 0)]),
                    o, filters=[(3, wg.OP_LT, 7)], threads=8)
        assert_groups_equal(g.export(), o.export(), ["sum_i", "count", "min_f", "max_f"])
        g.close()


def test_without_a_spill_budget_the_ledger_refuses():
    """The same query with no pinned spill budget fails with memory.ErrMemoryExceeded's code."""
    import torch
    import wadjet_b200 as wg
    with wg.Context(0, hbm_budget=64 * MB, pinned_spill=0) as ctx:
        k = torch.arange(1 << 21, dtype=torch.int64, device="cuda")
        g = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_COUNT, -1)], ndv_hint=1 << 21)
        with pytest.raises(wg.MemoryExceeded):
            wg.run_pipeline(ctx, wg.Batch([wg.Column(I64, k)]), g, device=True)
        g.close()


def _dev_words(valid):
    """LSB-first validity words of a bool mask, on the device."""
    import torch
    n = len(valid)
    bits = np.packbits(np.asarray(valid, bool), bitorder="little")
    words = np.zeros((n + 63) // 64 * 8, np.uint8)
    words[: len(bits)] = bits
    return torch.from_numpy(words.view(np.uint64)).cuda()


def test_spilled_aggregate_with_nulls_and_a_selection_matches_oracle():
    """NULLs in the key and in the aggregated columns, and a selection vector, under an 80 MB budget
    (the full table takes 84 MB): the selected rows are gathered, each nullable column's validity
    travels with the rows as one flag per row and is packed again per partition, and NULL keys form
    one group (aggregate_partial_spill.go spills partial state with selections and NULLs upstream).
    Two consume calls; the second has no NULLs in the value column."""
    import torch
    import wadjet_b200 as wg
    rng = np.random.default_rng(9)
    n = 1 << 21
    hk = rng.integers(0, 1 << 20, n).astype(np.int64) * 7919 - 12345
    hv = rng.integers(-10**6, 10**6, n).astype(np.int64)
    hf = rng.random(n)
    kvalid = rng.random(n) > 0.03
    vvalid = rng.random(n) > 0.1
    vvalid[n // 2:] = True
    sel = np.sort(rng.choice(n, size=n * 3 // 4, replace=False)).astype(np.uint32)
    budget = 80 * MB
    kinds = ["sum_i", "count", "min_f", "max_f"]
    with wg.Context(0, hbm_budget=budget, pinned_spill=1 << 30) as ctx:
        aggs = [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, 1), wg.AggColumn(wg.AGG_MIN, 2),
                wg.AggColumn(wg.AGG_MAX, 2)]
        g = wg.HashAggregate(ctx, [0], aggs, ndv_hint=1 << 20)
        half = n // 2
        for lo, hi in ((0, half), (half, n)):
            s = sel[(sel >= lo) & (sel < hi)] - lo
            vv = _dev_words(vvalid[lo:hi]) if lo == 0 else None
            cols = [wg.Column(I64, torch.from_numpy(hk[lo:hi]).cuda(), _dev_words(kvalid[lo:hi])),
                    wg.Column(I64, torch.from_numpy(hv[lo:hi]).cuda(), vv),
                    wg.Column(F64, torch.from_numpy(hf[lo:hi]).cuda())]
            wg.run_pipeline(ctx, wg.Batch(cols, sel=torch.from_numpy(s.astype(np.int32)).cuda()), g, device=True)
        g.finalize()
        assert ctx.ledger()["peak"] <= budget
        got = g.export()
        g.close()
    o = ob.Agg([0], [(0, 1, 0), (1, 1, 0), (2, 2, 0), (3, 2, 0)])
    # the oracle's pipeline takes flat batches: the selected rows themselves
    ob.pipeline(ob.HostBatch([(I64, hk[sel], kvalid[sel], 0), (I64, hv[sel], vvalid[sel], 0), (F64, hf[sel], None, 0)]),
                o, threads=8)
    want = o.export()
    assert (want["key_valid"][0] == 0).any()  # the NULL-key group exists
    assert_groups_equal(got, want, kinds)
