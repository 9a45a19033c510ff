"""LEFT, SEMI and ANTI joins against the oracle (exec.JoinType, join.go:20-30).

- LEFT: every probe row; an unmatched row (a NULL key included) once, with its
  build columns NULL (the generic probe's NULL-padded matchPair, join.go:3180).
- SEMI: a probe row with at least one match, once (executeSemiAntiJoin,
  join.go:3247); a NULL key never matches.
- ANTI: a probe row without a match, NULL keys included (join.go:3290).

Both the standalone bounded probe (pairs, with build row -1 where the output
has none, and the NULL gather of that row) and the fused filter → probe →
aggregate kernel are checked, on duplicate and unique build keys, with NULL
keys on both sides and with a selection vector.
"""
import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import assert_groups_equal, random_valid

pytestmark = pytest.mark.gpu

I32, I64, F64 = 1, 2, 4
TYPES = {"left": 1, "semi": 5, "anti": 6}


def _data(seed, dups, nulls, kt):
    rng = np.random.default_rng(seed)
    nb, npr = 20_000, 60_000
    dt = np.int32 if kt == I32 else np.int64
    bkeys = (rng.integers(0, 8_000, nb) if dups else rng.permutation(1 << 20)[:nb]).astype(dt)
    pkeys = bkeys[rng.integers(0, nb, npr)].copy()
    pkeys[::5] += 3  # some misses
    bvalid = random_valid(rng, nb, nulls)
    pvalid = random_valid(rng, npr, nulls)
    grp = rng.integers(0, 50, nb).astype(np.int32)
    val = rng.integers(-1000, 1000, npr).astype(np.int64)
    flt = rng.integers(0, 10, npr).astype(np.int32)
    return bkeys, bvalid, grp, pkeys, pvalid, val, flt


@pytest.mark.parametrize("jt", ["left", "semi", "anti"])
@pytest.mark.parametrize("kt", [I32, I64])
@pytest.mark.parametrize("dups,nulls", [(False, 0.0), (True, 0.0), (True, 0.05)])
def test_probe_pairs_match_oracle(ctx, jt, kt, dups, nulls):
    import wadjet_b200 as wg
    bkeys, bvalid, grp, pkeys, pvalid, _, _ = _data(31 + kt + 2 * dups, dups, nulls, kt)
    npay = [1] if jt == "left" else []
    j = wg.HashJoin(ctx, 0, 0, payload=npay, join_type=TYPES[jt])
    j.build([wg.Batch([wg.Column(kt, bkeys, bvalid), wg.Column(I32, grp)])])
    oj = ob.Join(1024, TYPES[jt])
    oj.append(kt, bkeys, bvalid)
    rng = np.random.default_rng(3)
    sel = np.sort(rng.choice(len(pkeys), size=len(pkeys) // 3, replace=False)).astype(np.uint32)
    for s in (None, sel):
        want = sorted(zip(*[a.tolist() for a in oj.probe(kt, pkeys, pvalid, sel=s)]))
        got = []
        for pr, br in j.probe(wg.Batch([wg.Column(kt, pkeys, pvalid)], sel=s), cap=9_999):
            got += list(zip(pr.tolist(), br.tolist()))
        assert sorted(got) == want
        if jt == "left":
            # gather: NULL where there is no build row, the payload elsewhere
            brows = np.array([b for _, b in got], np.int64)
            vals, ok = j.gather(0, brows, np.int32)
            np.testing.assert_array_equal(ok, brows >= 0)
            np.testing.assert_array_equal(vals[brows >= 0], grp[brows[brows >= 0]])
            assert (brows < 0).any()
    j.close()


def test_semi_and_anti_partition_the_probe_rows(ctx):
    """SEMI and ANTI over the same build side split the probe rows exactly in two."""
    import wadjet_b200 as wg
    bkeys, bvalid, _, pkeys, pvalid, _, _ = _data(5, True, 0.05, I64)
    rows = {}
    for jt in ("semi", "anti"):
        j = wg.HashJoin(ctx, 0, 0, join_type=TYPES[jt])
        j.build([wg.Batch([wg.Column(I64, bkeys, bvalid)])])
        rows[jt] = np.concatenate([pr for pr, _ in j.probe(wg.Batch([wg.Column(I64, pkeys, pvalid)]))])
        j.close()
    both = np.sort(np.concatenate([rows["semi"], rows["anti"]]))
    np.testing.assert_array_equal(both, np.arange(len(pkeys), dtype=np.uint32))


@pytest.mark.parametrize("jt", ["left", "semi", "anti"])
@pytest.mark.parametrize("dups,nulls", [(False, 0.0), (True, 0.05)])
def test_fused_pipeline_matches_oracle(ctx, jt, dups, nulls):
    """WHERE flt < 7, probe, GROUP BY (build grp for LEFT, else the probe value's sign
    class): COUNT(*), SUM(val), and for LEFT COUNT(grp) which skips the NULL-padded rows."""
    import wadjet_b200 as wg
    bkeys, bvalid, grp, pkeys, pvalid, val, flt = _data(77 + dups, dups, nulls, I32)
    left = jt == "left"
    j = wg.HashJoin(ctx, 0, 0, payload=[1] if left else [], join_type=TYPES[jt])
    j.build([wg.Batch([wg.Column(I32, bkeys, bvalid), wg.Column(I32, grp)])])
    oj = ob.Join(1024, TYPES[jt])
    oj.append(I32, bkeys, bvalid)
    batch = [(I32, pkeys, pvalid, 0), (I64, val, None, 0), (I32, flt, None, 0)]
    if left:
        key, aggs = [3], [(1, -1, 0), (0, 1, 0), (1, 3, 0)]
        kinds = ["count", "sum_i", "count"]
    else:
        key, aggs = [2], [(1, -1, 0), (0, 1, 0)]
        kinds = ["count", "sum_i"]
    g = wg.HashAggregate(ctx, key, [wg.AggColumn(f, c, o) for f, c, o in aggs], ndv_hint=64)
    wg.run_pipeline(ctx, wg.Batch([wg.Column(t, d, v) for t, d, v, _ in batch]), g, filters=[(2, wg.OP_LT, 7)],
                    join=j)
    g.finalize()
    o = ob.Agg(key, aggs)
    ob.pipeline(ob.HostBatch(batch), o, filters=[(2, wg.OP_LT, 7)], join=oj, probe_key=0,
                build=ob.HostBatch([(I32, bkeys, bvalid, 0), (I32, grp, None, 0)]),
                payload=[1] if left else [], threads=2)
    want = o.export()
    got = g.export()
    assert_groups_equal(got, want, kinds)
    if left:
        assert (want["key_valid"][0] == 0).any()  # the NULL-padded rows form the NULL group
    g.close()
    j.close()


@pytest.mark.parametrize("kt", [I32, I64])
@pytest.mark.parametrize("dups,nulls", [(False, 0.0), (True, 0.05)])
@pytest.mark.parametrize("use_sel", [False, True])
def test_bloom_filter_matches_oracle(ctx, kt, dups, nulls, use_sel):
    """BloomFilterOp.Execute (bloom_filter_op.go:39) over the probe keys, with the build side's
    bloom (HashJoin.buildBloom, join.go:1441): the same rows as the oracle's restatement, bit for
    bit (same hash, same sizing over the distinct keys), every true match among them."""
    import wadjet_b200 as wg
    bkeys, bvalid, _, pkeys, pvalid, _, _ = _data(41 + kt + dups, dups, nulls, kt)
    j = wg.HashJoin(ctx, 0, 0)
    j.build([wg.Batch([wg.Column(kt, bkeys, bvalid)])])
    oj = ob.Join(1024)
    oj.append(kt, bkeys, bvalid)
    rng = np.random.default_rng(2)
    sel = np.sort(rng.choice(len(pkeys), size=len(pkeys) // 2, replace=False)).astype(np.uint32) if use_sel else None
    got = j.bloom_filter(wg.Batch([wg.Column(kt, pkeys, pvalid)], sel=sel))
    want, _ = oj.bloom_filter(kt, pkeys, pvalid, sel=sel)
    np.testing.assert_array_equal(got, want)
    matched = np.unique(oj.probe(kt, pkeys, pvalid, sel=sel)[0])
    assert np.isin(matched, got).all()  # no false negatives
    assert len(got) < (len(sel) if use_sel else len(pkeys))  # the misses (key + 3) are mostly rejected
    j.close()


@pytest.mark.parametrize("jt", ["left", "semi", "anti"])
def test_fused_pipeline_with_bloom_matches_oracle(ctx, jt, monkeypatch):
    """The fused probe with the bloom checked before the hash index (WG_JOIN_BLOOM=1): the
    same groups as without it."""
    monkeypatch.setenv("WG_JOIN_BLOOM", "1")
    test_fused_pipeline_matches_oracle(ctx, jt, True, 0.05)
