"""The multi-rank path on CPU: two gloo ranks each aggregate a shard of the star
join, route their partial groups to owner ranks by the key's route hash
(partitionFor, partitioned_agg.go:221), exchange them with the same all-to-all
protocol the device path uses (exchange.exchange_rows) and merge what they own.
The union of the owned groups must equal one aggregate over the whole table
(partitioned_agg_test.go:91 'parallel = serial', with ranks in place of
workers), and every rank must own exactly the groups the route hash gives it."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_ROWS = 1 << 18


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_starjoin(row0: int, n: int):
    from oracle import binding as ob
    fk, qty, price, disc = ob.gen_starjoin_fact(n, row0=row0, threads=2)
    key, grp = ob.gen_starjoin_dim()
    j = ob.Join(1 << 22)
    j.append(1, key)
    agg = ob.Agg([4], [(0, 5, 0), (0, 2, 0), (1, -1, 0), (2, 3, 0), (3, 1, 0)])
    ob.pipeline(ob.HostBatch([(1, fk, None, 0), (1, qty, None, 0), (17, price, None, 2), (4, disc, None, 0)]), agg,
                filters=[(1, 4, 10)], join=j, probe_key=0, build=ob.HostBatch([(1, key, None, 0), (1, grp, None, 0)]),
                payload=[1], exprs=[ob.expr(4, [("col", 2), ("cf", 1.0), ("col", 3), "-", "*"])], threads=2)
    return agg.export()


KINDS = ["sum_f", "sum_d", "count", "min_f", "max_i"]


def _rank_main(rank: int, world: int, port: int, out_path: str):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import datetime
    from wadjet_b200.exchange import exchange_export, merge_exports, partition_for, route_hash_int, shard_range
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    row0, n = shard_range(N_ROWS, rank, world)
    part = _oracle_starjoin(row0, n)
    owned = exchange_export(dist, part, KINDS)
    # every group this rank finished is one the route hash assigns to it
    assert (partition_for(route_hash_int(owned["keys"][0]), world) == rank).all()
    parts = [None] * world
    dist.all_gather_object(parts, owned)
    if rank == 0:
        # owned key ranges are disjoint, so concatenating them is the whole result
        merged = merge_exports(parts, KINDS)
        assert merged["keys"].shape[1] == sum(p["keys"].shape[1] for p in parts)
        np.savez(out_path, **{k: merged[k] for k in ("keys", "key_valid", "count", "i64", "f64", "has")},
                 dec_hi=merged["dec"]["hi"], dec_lo=merged["dec"]["lo"])
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_merge_equals_serial(tmp_path):
    import sys
    sys.path.insert(0, ROOT)
    from tests.helpers import DEC_DTYPE, assert_groups_equal
    out = str(tmp_path / "merged.npz")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    z = np.load(out)
    got = {k: z[k] for k in ("keys", "key_valid", "count", "i64", "f64", "has")}
    got["dec"] = np.zeros(z["dec_hi"].shape, DEC_DTYPE)
    got["dec"]["hi"], got["dec"]["lo"] = z["dec_hi"], z["dec_lo"]
    want = _oracle_starjoin(0, N_ROWS)
    assert_groups_equal(got, want, KINDS)


def test_shard_ranges_cover_the_table():
    from wadjet_b200.exchange import shard_range
    for world in (1, 2, 3, 8):
        spans = [shard_range(1_000_003, r, world) for r in range(world)]
        assert spans[0][0] == 0
        for (a0, an), (b0, _) in zip(spans, spans[1:]):
            assert a0 + an == b0 and b0 % 64 == 0
        assert spans[-1][0] + spans[-1][1] == 1_000_003


@pytest.mark.parametrize("kind", ["min_d", "max_d", "sum_i"])
def test_merge_exports_decimal_and_wrapping(kind):
    from tests.helpers import DEC_DTYPE
    from wadjet_b200.exchange import merge_exports

    def part(keys, vals):
        n = len(keys)
        dec = np.zeros((1, n), DEC_DTYPE)
        for i, v in enumerate(vals):
            dec[0, i] = (-1 if v < 0 else 0, v & (2**64 - 1))
        i64 = np.array([[v if -2**63 <= v < 2**63 else 0 for v in vals]], np.int64)
        return {"keys": np.array([keys], np.int64), "key_valid": np.ones((1, n), np.uint8),
                "count": np.ones((1, n), np.int64), "i64": i64, "f64": np.zeros((1, n)), "dec": dec,
                "has": np.ones((1, n), np.uint8)}

    m = merge_exports([part([1, 2], [-5, 7]), part([1, 3], [4, 2**62])], [kind])
    keys = m["keys"][0].tolist()
    if kind == "sum_i":
        assert m["i64"][0][keys.index(1)] == -1
    else:
        d = m["dec"][0][keys.index(1)]
        assert (int(d["hi"]), int(d["lo"])) == ((-1, 2**64 - 5) if kind == "min_d" else (0, 4))


def test_partition_for_matches_multiply_shift():
    """partitionFor is hi64(hash * parts): the numpy form equals exact integer arithmetic."""
    from wadjet_b200.exchange import partition_for, route_hash_int
    rng = np.random.default_rng(3)
    keys = rng.integers(-2**63, 2**63 - 1, 10000, dtype=np.int64)
    h = route_hash_int(keys)
    for parts in (1, 2, 3, 7, 8, 96):
        want = [(int(x) * parts) >> 64 for x in h.tolist()]
        np.testing.assert_array_equal(partition_for(h, parts), want)
        assert ((partition_for(h, parts) >= 0) & (partition_for(h, parts) < parts)).all()
    # fibHash is the multiply by the golden-ratio constant mod 2^64
    assert int(route_hash_int(np.array([3]))[0]) == (3 * 11400714819323198485) % 2**64
