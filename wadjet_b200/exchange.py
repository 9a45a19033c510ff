"""Partial-aggregate exchange between ranks (one process per GPU).

Each rank aggregates its own shard of the fact table. The per-group partial
states are then hash-partitioned by owner rank and exchanged with one
all-to-all, so every rank finishes a disjoint key range: the same split as
partitionFor (internal/engine/exec/partitioned_agg.go:221, Lemire's
multiply-shift over the key's route hash) and the distributed shuffle
(internal/worker/partitioned_shuffle_sink.go:1039). Received states combine
the way MergeSink combines worker clones (exec/aggregate.go:4682 →
kernel.Accumulator.Merge, exec/kernel/types.go:106).

Two forms share one exchange protocol (`exchange_rows`: an all-to-all of the
row counts, then an all-to-all of the rows):

- `exchange_aggregate`: the device path. Partitioning and merging run on the
  GPU through the C ABI (wg_agg_partition_state / wg_agg_merge_state); the rows
  travel between HBMs over NCCL.
- `exchange_export`: the same protocol over exported group tables (numpy), used
  where no GPU is present (gloo ranks on CPU); owners come from the same route
  hash, merging from `merge_exports`.
"""
from __future__ import annotations

import numpy as np

DEC_DTYPE = np.dtype([("hi", "<i8"), ("lo", "<u8")])
_M128 = (1 << 128) - 1
_M64 = (1 << 64) - 1
FIB = 0x9E3779B97F4A7C15              # fibHash multiplier (exec/int_hash.go:95)
ROUTE_NULL_HASH = 0x9AE16A3B2F90404F  # routeNullHash (exec/partitioned_agg.go:197)


def shard_range(n_total: int, rank: int, world: int, align: int = 64) -> tuple[int, int]:
    """Rows [row0, row0 + n) of an n_total-row table owned by `rank` (aligned cuts)."""
    per = (n_total // world // align) * align
    row0 = rank * per
    n = n_total - row0 if rank == world - 1 else per
    return row0, n


# ------------------------------------------------------------------ routing --
def _mul_hi64(a: np.ndarray, b: int) -> np.ndarray:
    """High 64 bits of a * b for uint64 a and 0 <= b < 2^32 (bits.Mul64's hi word)."""
    a = a.astype(np.uint64)
    lo = (a & np.uint64(0xFFFFFFFF)) * np.uint64(b)
    hi = (a >> np.uint64(32)) * np.uint64(b)
    return (hi + (lo >> np.uint64(32))) >> np.uint64(32)


def partition_for(route_hash: np.ndarray, parts: int) -> np.ndarray:
    """partitionFor(hash, parts) = hi64(hash * parts) (partitioned_agg.go:221)."""
    return _mul_hi64(np.asarray(route_hash, np.uint64), parts).astype(np.int64)


def route_hash_int(keys: np.ndarray, valid: np.ndarray | None = None) -> np.ndarray:
    """routeHashInt64/Int32 (partitioned_agg.go:508-520): fibHash of the key widened to int64."""
    with np.errstate(over="ignore"):
        h = np.asarray(keys, np.int64).astype(np.uint64) * np.uint64(FIB)
    if valid is not None:
        h = np.where(np.asarray(valid).astype(bool), h, np.uint64(ROUTE_NULL_HASH))
    return h


def route_hash_packed(lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """packedHash(lo, hi) (exec/packed_hash.go:155), the routeHashPacked hash."""
    out = np.empty(len(lo), np.uint64)
    for i, (l, h) in enumerate(zip(np.asarray(lo, np.uint64).tolist(), np.asarray(hi, np.uint64).tolist())):
        a, b = l ^ FIB, h ^ 0x517CC1B727220A95
        p = a * b
        out[i] = ((p >> 64) ^ (p & _M64) ^ ((l + h) & _M64)) & _M64
    return out


def pack_key_words(keys: np.ndarray, layout, key_valid: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
    """(lo, hi) packed words of unpacked key columns, placed as buildPackedLayout does
    (exec/packed_hash.go:386); `layout` carries key_word / key_shift / key_i32 per column.
    A NULL column (key_valid 0) contributes no value bits."""
    lo = np.zeros(keys.shape[1], np.uint64)
    hi = np.zeros(keys.shape[1], np.uint64)
    for k in range(keys.shape[0]):
        v = keys[k].astype(np.int64)
        if key_valid is not None:
            v = np.where(key_valid[k].astype(bool), v, 0)
        w = (v.astype(np.uint32).astype(np.uint64) << np.uint64(layout.key_shift[k])) if layout.key_i32[k] \
            else v.astype(np.uint64)
        if layout.key_word[k] == 0:
            lo |= w
        else:
            hi |= w
    return lo, hi


# ---------------------------------------------------------------- protocol --
def exchange_rows(dist, rows, part_rows: list[int]):
    """All-to-all of state rows: `rows` (n, W) int64 grouped by destination rank,
    part_rows[r] rows for rank r. Returns (received rows, rows received from each rank).
    Every rank takes the same two collectives in the same order."""
    import torch
    send_counts = torch.tensor(part_rows, dtype=torch.int64, device=rows.device)
    recv_counts = torch.empty_like(send_counts)
    dist.all_to_all_single(recv_counts, send_counts)
    rc = [int(x) for x in recv_counts.tolist()]
    recv = torch.empty((sum(rc), rows.shape[1]), dtype=rows.dtype, device=rows.device)
    dist.all_to_all_single(recv, rows.contiguous(), rc, list(part_rows))
    return recv, rc


def _layout_to_tensor(lay, device):
    import ctypes as C
    import torch
    from . import _abi
    buf = np.frombuffer(C.string_at(C.addressof(lay), C.sizeof(_abi.wg_state_layout)), np.int32).copy() \
        if lay is not None else np.zeros(C.sizeof(_abi.wg_state_layout) // 4, np.int32)
    return torch.from_numpy(np.concatenate([[1 if lay is not None else 0], buf]).astype(np.int32)).to(device)


def _tensor_to_layout(t):
    import ctypes as C
    from . import _abi
    a = t.cpu().numpy().astype(np.int32)
    if a[0] == 0:
        return None
    lay = _abi.wg_state_layout()
    C.memmove(C.addressof(lay), a[1:].tobytes(), C.sizeof(lay))
    return lay


def exchange_aggregate(dist, local, owner) -> None:
    """Device path: hash-partition `local`'s finalized groups by owner rank, exchange
    them over the process group, and merge what this rank owns into `owner` (an
    aggregate of the same shape that is not finalized)."""
    import torch
    world = dist.get_world_size()
    rows, part_rows = local.partition_state(world)
    lay = local.state_layout() if sum(part_rows) else None
    device = rows.device
    # each rank's row layout (ranks that saw NULLs carry null counters others lack)
    mine = _layout_to_tensor(lay, device)
    alls = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(alls, mine)
    layouts = [_tensor_to_layout(t) for t in alls]
    width = torch.tensor([rows.shape[1] if lay is not None else 1], dtype=torch.int64, device=device)
    dist.all_reduce(width, op=dist.ReduceOp.MAX)
    w = int(width.item())
    if rows.shape[1] < w:
        rows = torch.nn.functional.pad(rows, (0, w - rows.shape[1]))
    recv, rc = exchange_rows(dist, rows, part_rows)
    torch.cuda.current_stream(device).synchronize()
    off = 0
    for r in range(world):
        if rc[r]:
            src = layouts[r]
            owner.merge_state(src, recv[off:off + rc[r], :1 + src.slot_words].contiguous())
        off += rc[r]


# ------------------------------------------------------- exported (numpy) form --
_FIELDS = ("count", "i64", "f64", "dec_hi", "dec_lo", "has")


def _owners(part: dict, world: int, layout=None) -> np.ndarray:
    nk = part["keys"].shape[0]
    n = part["keys"].shape[1]
    if nk == 0:
        return np.zeros(n, np.int64)
    valid = part["key_valid"].all(axis=0)
    if nk == 1:
        h = route_hash_int(part["keys"][0], part["key_valid"][0])
    else:
        lo, hi = pack_key_words(part["keys"], layout)
        h = np.where(valid, route_hash_packed(lo, hi), np.uint64(ROUTE_NULL_HASH))
    return partition_for(h, world)


def _pack(part: dict, order: np.ndarray) -> np.ndarray:
    nk = part["keys"].shape[0]
    na = part["count"].shape[0]
    cols = [part["key_valid"][k].astype(np.int64)[order] for k in range(nk)]
    cols += [part["keys"][k].astype(np.int64)[order] for k in range(nk)]
    for a in range(na):
        cols += [part["count"][a][order], part["i64"][a][order], part["f64"][a].view(np.int64)[order],
                 part["dec"][a]["hi"][order], part["dec"][a]["lo"].view(np.int64)[order],
                 part["has"][a].astype(np.int64)[order]]
    return np.stack(cols, axis=1) if cols else np.zeros((len(order), 0), np.int64)


def _unpack(rows: np.ndarray, nk: int, na: int) -> dict:
    n = rows.shape[0]
    r = {"key_valid": np.zeros((nk, n), np.uint8), "keys": np.zeros((nk, n), np.int64)}
    for k in range(nk):
        r["key_valid"][k] = rows[:, k]
        r["keys"][k] = rows[:, nk + k]
    r["count"] = np.zeros((na, n), np.int64)
    r["i64"] = np.zeros((na, n), np.int64)
    r["f64"] = np.zeros((na, n), np.float64)
    r["dec"] = np.zeros((na, n), DEC_DTYPE)
    r["has"] = np.zeros((na, n), np.uint8)
    for a in range(na):
        b = 2 * nk + 6 * a
        r["count"][a] = rows[:, b]
        r["i64"][a] = rows[:, b + 1]
        r["f64"][a] = rows[:, b + 2].view(np.float64)
        r["dec"][a]["hi"] = rows[:, b + 3]
        r["dec"][a]["lo"] = rows[:, b + 4].view(np.uint64)
        r["has"][a] = rows[:, b + 5]
    return r


def exchange_export(dist, part: dict, kinds: list[str], layout=None) -> dict:
    """The exchange over an exported group table (HashAggregate.export() layout):
    groups routed to their owner rank by the route hash, exchanged with
    `exchange_rows`, and merged; returns the groups this rank owns."""
    import torch
    world = dist.get_world_size()
    nk, na = part["keys"].shape[0], part["count"].shape[0]
    owners = _owners(part, world, layout)
    order = np.argsort(owners, kind="stable")
    counts = np.bincount(owners, minlength=world).tolist()
    rows = torch.from_numpy(np.ascontiguousarray(_pack(part, order)))
    recv, rc = exchange_rows(dist, rows, counts)
    got = recv.numpy()
    parts, off = [], 0
    for r in range(world):
        parts.append(_unpack(got[off:off + rc[r]], nk, na))
        off += rc[r]
    return merge_exports(parts, kinds)


# ------------------------------------------------------------------- merging --
def _dec_to_int(d: np.ndarray) -> list[int]:
    # Go's Int128{Hi, Lo} as one two's-complement integer: Python's shift and OR of
    # a signed hi word already give the signed value
    return [(int(h) << 64) | int(l) for h, l in zip(d["hi"], d["lo"])]


def _int_to_dec(vals: list[int]) -> np.ndarray:
    out = np.zeros(len(vals), DEC_DTYPE)
    for i, v in enumerate(vals):
        v &= _M128
        hi = v >> 64
        out[i]["hi"] = hi - (1 << 64) if hi >= (1 << 63) else hi
        out[i]["lo"] = v & _M64
    return out


def merge_exports(parts: list[dict], kinds: list[str]) -> dict:
    """Combine exported group tables (HashAggregate.export() layout) of several ranks.

    kinds[a] names aggregate a's state: count | sum_i | sum_f | sum_d | min_i | max_i | min_f | max_f |
    min_d | max_d | avg_i | avg_f | avg_d.
    """
    nk = parts[0]["keys"].shape[0]
    na = len(kinds)
    keys = np.concatenate([p["keys"] for p in parts], axis=1)
    kv = np.concatenate([p["key_valid"] for p in parts], axis=1)
    n = keys.shape[1]
    if nk:
        ident = np.stack([kv[k] for k in range(nk)] + [np.where(kv[k] != 0, keys[k], 0) for k in range(nk)], axis=1)
        uniq, inv = np.unique(ident, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        g = uniq.shape[0]
        out_kv = uniq[:, :nk].T.astype(np.uint8)
        out_keys = uniq[:, nk:].T.astype(np.int64)
    else:
        g, inv = (1 if n else 0), np.zeros(n, np.int64)
        out_kv = np.zeros((0, g), np.uint8)
        out_keys = np.zeros((0, g), np.int64)
    cat = {f: np.concatenate([p[f] for p in parts], axis=1) for f in ("count", "i64", "f64", "dec", "has")}
    r = {"keys": out_keys, "key_valid": out_kv, "count": np.zeros((na, g), np.int64),
         "i64": np.zeros((na, g), np.int64), "f64": np.zeros((na, g), np.float64),
         "dec": np.zeros((na, g), DEC_DTYPE), "has": np.zeros((na, g), np.uint8)}
    for a, kind in enumerate(kinds):
        np.add.at(r["count"][a], inv, cat["count"][a])
        has = cat["has"][a].astype(bool)
        hg = np.zeros(g, bool)
        np.logical_or.at(hg, inv, has)
        r["has"][a] = hg if kind.startswith(("min", "max")) else (r["count"][a] > 0)
        if kind in ("sum_i", "avg_i"):
            with np.errstate(over="ignore"):
                np.add.at(r["i64"][a], inv, cat["i64"][a])
        elif kind in ("sum_f", "avg_f"):
            np.add.at(r["f64"][a], inv, cat["f64"][a])
        elif kind in ("sum_d", "avg_d"):
            acc = [0] * g
            for i, v in zip(inv.tolist(), _dec_to_int(cat["dec"][a])):
                acc[i] += v
            r["dec"][a] = _int_to_dec(acc)
        elif kind in ("min_i", "max_i", "min_f", "max_f"):
            f = "i64" if kind.endswith("_i") else "f64"
            lo = kind.startswith("min")
            fill = (np.iinfo(np.int64).max if lo else np.iinfo(np.int64).min) if f == "i64" else (np.inf if lo else -np.inf)
            acc = np.full(g, fill, dtype=r[f].dtype)
            vals = np.where(has, cat[f][a], fill)
            (np.minimum if lo else np.maximum).at(acc, inv, vals)
            r[f][a] = np.where(hg, acc, 0)
        elif kind in ("min_d", "max_d"):
            best: list = [None] * g
            for i, v, h in zip(inv.tolist(), _dec_to_int(cat["dec"][a]), has.tolist()):
                if not h:
                    continue
                s = v - (1 << 128) if v >= (1 << 127) else v
                if best[i] is None or (s < best[i] if kind == "min_d" else s > best[i]):
                    best[i] = s
            r["dec"][a] = _int_to_dec([0 if b is None else b for b in best])
    return r
