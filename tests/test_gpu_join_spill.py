"""The partitioned (grace) join build under an HBM cap, against the oracle.

When the ledger refuses the build side's columns or its index, the build rows
move to host memory in 64 key-hash partitions (join_partition_arrival.go:48
builds partitioned on arrival and spills a partition at a time); the fused
pipeline then probes in passes over groups of partitions that fit, each probe
row taking part in its key's pass. The result must equal the oracle's, for
every join type, int32 and int64 keys, duplicate keys and NULLs on both sides,
over several pipeline calls, as join_spill_test.go checks the spilled join
against the in-memory one.
"""
import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import assert_groups_equal, random_valid

pytestmark = pytest.mark.gpu

I32, I64 = 1, 2
TYPES = {"inner": 0, "left": 1, "semi": 5, "anti": 6}
CAP = 16 << 20  # the build (1M rows) and its index need 25-50 MB


def _data(seed, dups, nulls, kt):
    rng = np.random.default_rng(seed)
    nb, npr = 1_000_000, 3_000_000
    dt = np.int32 if kt == I32 else np.int64
    span = 300_000 if dups else 1 << 40
    bkeys = (rng.integers(0, span, nb) if dups else rng.choice(1 << 30, nb, replace=False)).astype(dt)
    pkeys = bkeys[rng.integers(0, nb, npr)].copy()
    pkeys[::4] += 7  # some misses
    bvalid = random_valid(rng, nb, nulls)
    pvalid = random_valid(rng, npr, nulls)
    grp = rng.integers(0, 40, nb).astype(np.int32)
    gvalid = random_valid(rng, nb, nulls)
    val = rng.integers(-1000, 1000, npr).astype(np.int64)
    flt = rng.integers(0, 10, npr).astype(np.int32)
    return bkeys, bvalid, grp, gvalid, pkeys, pvalid, val, flt


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _dev_valid(v, n):
    """LSB-first validity words of a bool mask, on the device (None: no NULLs)."""
    if v is None:
        return None
    bits = np.packbits(np.asarray(v, bool), bitorder="little")
    words = np.zeros((n + 63) // 64 * 8, np.uint8)
    words[: len(bits)] = bits
    return _dev(words.view(np.uint64))


@pytest.mark.parametrize("jt", ["inner", "left", "semi", "anti"])
@pytest.mark.parametrize("kt,dups,nulls", [(I32, False, 0.0), (I64, True, 0.0), (I64, True, 0.05)])
def test_grace_join_matches_oracle(jt, kt, dups, nulls):
    """WHERE flt < 7, probe, GROUP BY (build grp for INNER/LEFT, else flt): COUNT(*),
    SUM(val), and for INNER/LEFT COUNT(grp), over two pipeline calls on device input."""
    import wadjet_b200 as wg
    bkeys, bvalid, grp, gvalid, pkeys, pvalid, val, flt = _data(11 + kt + dups, dups, nulls, kt)
    with_pay = jt in ("inner", "left")
    c = wg.Context(0, hbm_budget=CAP)
    j = wg.HashJoin(c, 0, 0, payload=[1] if with_pay else [], join_type=TYPES[jt], build_row_hint=len(bkeys))
    j.build([wg.Batch([wg.Column(kt, bkeys, bvalid), wg.Column(I32, grp, gvalid)])])
    assert j.stats() == (len(bkeys), -1)  # partitioned: distinct keys are not counted across partitions
    if with_pay:
        key, aggs, kinds = [3], [(1, -1, 0), (0, 1, 0), (1, 3, 0)], ["count", "sum_i", "count"]
    else:
        key, aggs, kinds = [2], [(1, -1, 0), (0, 1, 0)], ["count", "sum_i"]
    g = wg.HashAggregate(c, key, [wg.AggColumn(f, col, o) for f, col, o in aggs], ndv_hint=64)
    half = len(pkeys) // 2 // 64 * 64
    for r0, r1 in ((0, half), (half, len(pkeys))):
        pv = None if pvalid is None else pvalid[r0:r1]
        cols = [wg.Column(kt, _dev(pkeys[r0:r1]), _dev_valid(pv, r1 - r0)), wg.Column(I64, _dev(val[r0:r1])),
                wg.Column(I32, _dev(flt[r0:r1]))]
        wg.run_pipeline(c, wg.Batch(cols), g, filters=[(2, wg.OP_LT, 7)], join=j, device=True)
    g.finalize()
    assert c.ledger()["peak"] <= CAP
    oj = ob.Join(1024, TYPES[jt])
    oj.append(kt, bkeys, bvalid)
    o = ob.Agg(key, aggs)
    ob.pipeline(ob.HostBatch([(kt, pkeys, pvalid, 0), (I64, val, None, 0), (I32, flt, None, 0)]), o,
                filters=[(2, wg.OP_LT, 7)], join=oj, probe_key=0,
                build=ob.HostBatch([(kt, bkeys, bvalid, 0), (I32, grp, gvalid, 0)]),
                payload=[1] if with_pay else [], threads=8)
    assert_groups_equal(g.export(), o.export(), kinds)
    g.close()
    j.close()
    c.close()


def test_grace_join_refuses_the_standalone_probe():
    import wadjet_b200 as wg
    bkeys, bvalid, grp, gvalid, pkeys, pvalid, _, _ = _data(3, False, 0.0, I64)
    c = wg.Context(0, hbm_budget=CAP)
    j = wg.HashJoin(c, 0, 0, payload=[1])
    j.build([wg.Batch([wg.Column(I64, bkeys), wg.Column(I32, grp)])])
    with pytest.raises(wg.WadjetGPUError) as ei:
        next(j.probe(wg.Batch([wg.Column(I64, pkeys[:1000])])))
    assert ei.value.status == wg._abi.WG_E_UNSUPPORTED
    # a reset forgets the partitions; a small build then fits the device again
    j.reset()
    j.build([wg.Batch([wg.Column(I64, bkeys[:1000]), wg.Column(I32, grp[:1000])])])
    assert j.stats()[1] == 1000
    j.close()
    c.close()
