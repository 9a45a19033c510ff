"""Autotuner for the batched mode's launch shape and table sizing.

Searches wg_tune_params (rows per work item, threads per CTA, CTAs per SM, the
group count below which a query pre-combines each work item in shared memory,
and the table load the ndv hint is sized for) on a representative sample of the
batched workload, times each candidate as the median of replays of its captured
graph, and writes the fastest to wadjet_b200/tuned/batched.json, which
``load_tuned()`` hands to ``BatchedQueries``.

Run on a GPU: python -m wadjet_b200.autotune [--queries 128] [--max-rows 2000000]
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import statistics
import time

HERE = os.path.dirname(os.path.abspath(__file__))
TUNED = os.path.join(HERE, "tuned", "batched.json")

GRID = {
    "tile_rows": [8192, 32768, 131072],
    "block": [256, 512],
    "ctas_per_sm": [1, 2, 4],
    "smem_max_groups": [-1, 1024, 8192],
    "max_load": [0.5],
}


def load_tuned():
    """The persisted choice as TuneParams, or None when the tuner has not run."""
    from . import TuneParams
    try:
        with open(TUNED) as f:
            p = json.load(f)["params"]
        return TuneParams(**p)
    except (OSError, KeyError, ValueError, TypeError):
        return None


def sample_queries(ctx, nq: int, max_rows: int):
    import wadjet_b200 as wg
    from wadjet_b200 import synth
    qs = []
    for q in range(nq):
        n, card, thr = synth.batched_params(q)
        key, val, filt, card, thr = synth.batched_query(ctx, q, rows=min(n, max_rows))
        vt = wg.TYPE_INT64 if q % 2 == 0 else wg.TYPE_FLOAT64
        qs.append({"batch": wg.Batch([wg.Column(wg.TYPE_INT64, key), wg.Column(vt, val),
                                      wg.Column(wg.TYPE_INT32, filt)]),
                   "group_by": [0],
                   "aggs": [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1),
                            wg.AggColumn(wg.AGG_MIN, 1), wg.AggColumn(wg.AGG_MAX, 1)],
                   "filters": [(2, wg.OP_LT, thr)], "ndv_hint": card, "_keep": (key, val, filt)})
    return qs


def time_params(ctx, qs, params, reps: int = 5) -> float:
    import torch
    import wadjet_b200 as wg
    b = wg.BatchedQueries(ctx, qs, params)
    stream = torch.cuda.ExternalStream(ctx.stream)
    try:
        b.run()
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times)
    finally:
        b.close()


def tune(ctx, nq: int, max_rows: int, grid=None, log=print) -> dict:
    import wadjet_b200 as wg
    grid = grid or GRID
    qs = sample_queries(ctx, nq, max_rows)
    rows = sum(int(q["batch"].len) for q in qs)
    results = []
    names = list(grid)
    for combo in itertools.product(*[grid[k] for k in names]):
        p = dict(zip(names, combo))
        try:
            ms = time_params(ctx, qs, wg.TuneParams(**p))
        except wg.WadjetGPUError as e:  # a shape this device cannot launch: skip it
            log(json.dumps({"params": p, "skipped": str(e)}))
            continue
        results.append({"params": p, "ms": ms})
        log(json.dumps(results[-1]))
    best = min(results, key=lambda r: r["ms"])
    import torch
    out = {"params": best["params"], "best_ms": best["ms"], "sample_queries": nq, "sample_rows": rows,
           "device": torch.cuda.get_device_name(), "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
           "candidates": results}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--queries", type=int, default=128)
    ap.add_argument("--max-rows", type=int, default=2_000_000)
    ap.add_argument("--out", default=TUNED)
    a = ap.parse_args()
    import wadjet_b200 as wg
    with wg.Context(0) as ctx:
        res = tune(ctx, a.queries, a.max_rows)
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({"best": res["params"], "ms": res["best_ms"]}))


if __name__ == "__main__":
    main()
