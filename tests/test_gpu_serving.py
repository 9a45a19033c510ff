"""Serving loop: each request's result is the same alone and in a concurrent mix
(and equal to the oracle), and admission by the HBM ledger refuses a request
that can never fit instead of waiting forever."""
import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import assert_groups_equal

pytestmark = pytest.mark.gpu

I32, I64, F64, DEC = 1, 2, 4, 17


@pytest.fixture(scope="module")
def tables(ctx):
    import torch
    import wadjet_b200 as wg
    from wadjet_b200 import synth
    t = {}
    t["gb"] = synth.groupby(ctx, 1 << 20)
    t["fact"] = synth.starjoin_fact(ctx, 1 << 21)
    key, grp = synth.starjoin_dim(ctx)
    t["dim"] = (key, grp)
    join = wg.HashJoin(ctx, 0, 0, payload=[1], build_row_hint=1 << 22)
    join.build([wg.Batch([wg.Column(I32, key), wg.Column(I32, grp)])], device=True)
    t["join"] = join
    rng = np.random.default_rng(7)
    n = 1 << 20
    addr = (np.int64(10 << 24) + rng.integers(0, 1 << 24, n)).astype(np.int64)
    nbytes = np.round(rng.lognormal(8.0, 2.0, n)).astype(np.int64)
    t["ip"] = (torch.from_numpy(addr).cuda(), torch.from_numpy(nbytes).cuda())
    yield t
    join.close()


def templates(wg, t):
    gb = t["gb"]
    fk, qty, price, disc = t["fact"]
    addr, nbytes = t["ip"]
    return {
        "groupby": dict(batch=wg.Batch([wg.Column(I64, gb[0]), wg.Column(I64, gb[1]), wg.Column(F64, gb[2]),
                                        wg.Column(I32, gb[3])]),
                        group_by=[0], aggs=[wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1),
                                            wg.AggColumn(wg.AGG_MIN, 2), wg.AggColumn(wg.AGG_MAX, 2)],
                        filters=[(3, wg.OP_LT, 7)], ndv_hint=4096),
        "join": dict(batch=wg.Batch([wg.Column(I32, fk), wg.Column(I32, qty), wg.Column(DEC, price, scale=2),
                                     wg.Column(F64, disc)]),
                     group_by=[4], aggs=[wg.AggColumn(wg.AGG_SUM, 5), wg.AggColumn(wg.AGG_SUM, 2)],
                     filters=[(1, wg.OP_GT, 10)], join=t["join"],
                     exprs=[wg.Expr(F64, [wg.Expr.col(2), wg.Expr.const_f(1.0), wg.Expr.col(3), "-", "*"])],
                     ndv_hint=1000),
        "ipv4": dict(batch=wg.Batch([wg.Column(I64, addr), wg.Column(I64, nbytes)]),
                     group_by=[2], aggs=[wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1)],
                     exprs=[wg.Expr(I64, [wg.Expr.col(0), wg.Expr.const_i(8), ">>"])], ndv_hint=1 << 16),
    }


KINDS = {"groupby": ["sum_i", "count", "min_f", "max_f"], "join": ["sum_f", "sum_d"], "ipv4": ["sum_i", "count"]}


def test_same_result_alone_and_in_the_mix(ctx, tables):
    import wadjet_b200 as wg
    tpl = templates(wg, tables)
    alone = {}
    s1 = wg.Server(ctx, 1)
    for name, spec in tpl.items():
        t = s1.submit(**spec)
        n, _ = s1.wait(t)
        alone[name] = s1.export(t, n)
        s1.release(t)
    s1.close()
    s8 = wg.Server(ctx, 6)
    tickets = []
    order = ["groupby", "join", "ipv4"] * 10
    for name in order:
        tickets.append((name, s8.submit(**tpl[name])))
    for name, t in tickets:
        n, lat = s8.wait(t, timeout=120.0)
        assert lat > 0
        assert_groups_equal(s8.export(t, n), alone[name], KINDS[name])
        s8.release(t)
    st = s8.stats()
    assert st["completed"] == len(order) and st["failed"] == 0
    assert st["p99_s"] >= st["p50_s"] > 0
    s8.close()


def test_ipv4_template_matches_oracle(ctx, tables):
    import wadjet_b200 as wg
    tpl = templates(wg, tables)["ipv4"]
    s = wg.Server(ctx, 2)
    t = s.submit(**tpl)
    n, _ = s.wait(t)
    got = s.export(t, n)
    s.release(t)
    s.close()
    addr, nbytes = (x.cpu().numpy() for x in tables["ip"])
    o = ob.Agg([2], [(0, 1, 0), (1, -1, 0)])
    ob.pipeline(ob.HostBatch([(I64, addr, None, 0), (I64, nbytes, None, 0)]), o,
                exprs=[ob.expr(I64, [("col", 0), ("ci", 8), ">>"])], threads=4)
    assert_groups_equal(got, o.export(), KINDS["ipv4"])


def test_admission_refuses_what_never_fits(ctx, tables):
    import wadjet_b200 as wg
    tpl = templates(wg, tables)["groupby"]
    s = wg.Server(ctx, 2)
    budget = ctx.ledger()["budget"]
    t_big = s.submit(**tpl, est_bytes=budget * 2)
    with pytest.raises(wg.MemoryExceeded):
        s.wait(t_big, timeout=60.0)
    t_ok = s.submit(**tpl)
    n, _ = s.wait(t_ok, timeout=60.0)
    assert n == 4096
    s.release(t_big)
    s.release(t_ok)
    s.close()


def test_cancel_withdraws_queued_requests(ctx, tables):
    """A request still in the queue can be withdrawn (the caller's context was
    cancelled): its wait raises Cancelled, it never runs, and the requests ahead
    of it and after it finish with their usual results."""
    import wadjet_b200 as wg
    tpl = templates(wg, tables)
    s = wg.Server(ctx, 1)  # one slot: requests behind the first one stay queued
    ahead = [s.submit(**tpl["join"]) for _ in range(4)]
    doomed = [s.submit(**tpl["groupby"]) for _ in range(2)]
    after = s.submit(**tpl["ipv4"])
    for t in doomed:
        s.cancel(t)
    for t in doomed:
        with pytest.raises(wg.Cancelled):
            s.wait(t, timeout=60.0)
    for t in ahead:
        n, _ = s.wait(t, timeout=120.0)
        assert 990 <= n <= 1000
    n, _ = s.wait(after, timeout=120.0)
    assert 60000 < n <= 1 << 16
    with pytest.raises(wg.WadjetGPUError) as ei:
        s.cancel(after)  # finished requests cannot be cancelled
    assert ei.value.status == wg._abi.WG_E_STATE
    st = s.stats()
    assert st["cancelled"] == 2 and st["completed"] == 5 and st["failed"] == 0
    for t in ahead + doomed + [after]:
        s.release(t)
    s.close()


def test_large_requests_match_oracle_in_the_mix(ctx, tables):
    """Requests of 1.2 * 10^7 and 3 * 10^7 rows (the configured sizes reach 10^8) served
    beside small ones: each result equals the oracle's over the same rows."""
    import torch
    import wadjet_b200 as wg
    from wadjet_b200 import synth
    n = 30_000_000
    k, v, f, flag = synth.groupby(ctx, n)
    aggs = [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_MIN, 2),
            wg.AggColumn(wg.AGG_MAX, 2)]

    def spec(m):
        return dict(batch=wg.Batch([wg.Column(I64, k[:m]), wg.Column(I64, v[:m]), wg.Column(F64, f[:m]),
                                    wg.Column(I32, flag[:m])]), group_by=[0], aggs=aggs,
                    filters=[(3, wg.OP_LT, 7)], ndv_hint=4096)

    small = templates(wg, tables)
    s = wg.Server(ctx, 4)
    sizes = [12_000_000, n]
    big = [s.submit(**spec(m)) for m in sizes]
    others = [s.submit(**small[name]) for name in ("join", "ipv4", "groupby") * 3]
    hk, hv, hf, hflag = (t.cpu().numpy() for t in (k, v, f, flag))
    for m, t in zip(sizes, big):
        cnt, _ = s.wait(t, timeout=300.0)
        got = s.export(t, cnt)
        s.release(t)
        o = ob.Agg([0], [(0, 1, 0), (1, -1, 0), (2, 2, 0), (3, 2, 0)])
        ob.pipeline(ob.HostBatch([(I64, hk[:m], None, 0), (I64, hv[:m], None, 0), (F64, hf[:m], None, 0),
                                  (I32, hflag[:m], None, 0)]), o, filters=[(3, 2, 7)], threads=8)
        assert_groups_equal(got, o.export(), KINDS["groupby"])
    for t in others:
        s.wait(t, timeout=300.0)
        s.release(t)
    s.close()
    del k, v, f, flag
    torch.cuda.empty_cache()
