#!/usr/bin/env python
"""Star join + aggregate on one B200 (per rank): the filter → hash-join → hash-aggregate path.

Workload (synthetic, seeded; include/wadjet_synth.h): a 2^28-row fact table
(fk int32 Zipf(1.1) over 2^22 keys, qty int32 U[1,50], price DECIMAL(15,2) as
Int128, disc float64 U[0,0.1)) joined to a 2^22-row dimension (unique int32 key,
grp int32 U[0,1000)):

    SELECT grp, SUM(price*(1-disc)), SUM(price) FROM fact JOIN dim ON fk = key
    WHERE qty > 10 GROUP BY grp

One step = the whole query: build the join index from the dimension, run the
fused filter → probe → project → aggregate pass over every fact row, finalize
(compact the groups) and read the group count back. `value` is fact rows per
second with the inputs resident in HBM; `e2e` is the same query through the
public API from pinned host buffers (host→device copies and the result read
inside the timed region). Inputs (8.6 GB per rank) are far larger than the
126 MB L2, so no flush is needed between steps.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
For N > 1 launch with torchrun (one rank per GPU); ranks process disjoint fact
shards (weak scaling) and the per-group partial states are combined on rank 0
after an all-gather.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FACT_ROWS = 1 << 28
DIM_ROWS = 1 << 22
GROUPS = 1000
FACT_BYTES_PER_ROW = 4 + 4 + 16 + 8      # fk, qty, price (Int128), disc
DIM_BYTES_PER_ROW = 4 + 4                # key, grp
GROUP_STATE_BYTES = 8 + 8 + 16 + 8       # key, rows, SUM f64, SUM Int128
CPU_SAMPLE_ROWS = 1 << 24
METRIC = "rows/s (filter+join+hash-agg, star join 2^28 fact rows)"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--rows", type=int, default=FACT_ROWS)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for name, flag in zip(names, parts[5:9]):
                    if flag.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# -------------------------------------------------------------- reference --
def cpu_pipeline_sample(rows: int, threads: int, repeats: int = 1):
    """The oracle's Pipeline.Run (the reference algorithm restated in C++) on a
    host-resident sample of the same workload; returns rows/s of the best repeat."""
    import numpy as np
    from oracle import binding as ob
    fk, qty, price, disc = ob.gen_starjoin_fact(rows, threads=threads)
    key, grp = ob.gen_starjoin_dim(DIM_ROWS)
    build = ob.HostBatch([(1, key, None, 0), (1, grp, None, 0)])
    batch = ob.HostBatch([(1, fk, None, 0), (1, qty, None, 0), (17, price, None, 2), (4, disc, None, 0)])
    expr = ob.expr(4, [("col", 2), ("cf", 1.0), ("col", 3), "-", "*"])
    best = None
    for _ in range(repeats):
        t0 = time.perf_counter()
        j = ob.Join(DIM_ROWS)
        j.append(1, key)
        agg = ob.Agg([4], [(0, 5, 0), (0, 2, 0)])
        ob.pipeline(batch, agg, filters=[(1, 4, 10)], join=j, probe_key=0, build=build, payload=[1], exprs=[expr],
                    threads=threads)
        groups = agg.groups()
        dt = time.perf_counter() - t0
        assert groups == GROUPS, groups
        best = dt if best is None else min(best, dt)
    return rows / best, best


def run_reference(args, rank: int):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    times = []
    for i in range(args.warmup + args.steps):
        rps, dt = cpu_pipeline_sample(CPU_SAMPLE_ROWS, threads)
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = CPU_SAMPLE_ROWS * len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int128+f64", "data": "synthetic",
        "config": {"workload": "star join + aggregate (sample of 2^24 fact rows per step)", "fact_rows": CPU_SAMPLE_ROWS,
                   "dim_rows": DIM_ROWS, "groups": GROUPS, "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                         "sample": f"{CPU_SAMPLE_ROWS} fact rows per step (of the 2^28-row workload), "
                                   "C++ restatement of the reference's Pipeline.Run (Go toolchain absent)"},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------- ours --
def run_ours(args, rank: int, world: int, local_rank: int):
    import numpy as np
    import torch
    import wadjet_b200 as wg
    from wadjet_b200 import synth

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local_rank))
    ctx = wg.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local_rank))
    n = args.rows
    row0 = rank * n
    fk, qty, price, disc = synth.starjoin_fact(ctx, n, row0=row0, device=local_rank)
    key, grp = synth.starjoin_dim(ctx, DIM_ROWS, device=local_rank)
    torch.cuda.synchronize()

    I32, F64, DEC = wg.TYPE_INT32, wg.TYPE_FLOAT64, wg.TYPE_DECIMAL
    expr = wg.Expr(F64, [wg.Expr.col(2), wg.Expr.const_f(1.0), wg.Expr.col(3), "-", "*"])
    join = wg.HashJoin(ctx, 0, 0, payload=[1], build_row_hint=DIM_ROWS)
    agg = wg.HashAggregate(ctx, [4], [wg.AggColumn(wg.AGG_SUM, 5), wg.AggColumn(wg.AGG_SUM, 2)], ndv_hint=GROUPS)
    dim_dev = wg.Batch([wg.Column(I32, key), wg.Column(I32, grp)])
    fact_dev = wg.Batch([wg.Column(I32, fk), wg.Column(I32, qty), wg.Column(DEC, price, scale=2),
                         wg.Column(F64, disc)])
    kev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    kernel_ms = []

    def step(fact, dim, device: bool, time_kernel: bool = False):
        join.reset()
        join.build([dim], device=device)
        agg.reset()
        if time_kernel:
            kev[0].record(stream)
        wg.run_pipeline(ctx, fact, agg, filters=[(1, wg.OP_GT, 10)], join=join, exprs=[expr], device=device)
        if time_kernel:
            kev[1].record(stream)
        return agg.finalize()

    def combine_partials():
        """Per-group partial states of every rank, merged on rank 0 (the exchange step)."""
        e = agg.export()
        part = {"keys": e["keys"][0], "count": e["count"][0], "f64": e["f64"][0],
                "hi": e["dec"][1]["hi"], "lo": e["dec"][1]["lo"]}
        if dist is None:
            return part
        parts = [None] * world
        dist.all_gather_object(parts, part)
        if rank != 0:
            return None
        acc = {}
        for p in parts:
            for i, k in enumerate(p["keys"].tolist()):
                v = (int(p["hi"][i]) << 64) | int(p["lo"][i])
                a = acc.setdefault(k, [0, 0.0, 0])
                a[0] += int(p["count"][i]); a[1] += float(p["f64"][i]); a[2] += v
        return acc

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, k, w):
        for _ in range(w):
            fn()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        l0 = ctx.launches
        ev[0].record(stream)
        for _ in range(k):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        launches = ctx.launches - l0
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        return ms, launches

    # ---- device-resident query ------------------------------------------
    clocks = ClockSampler(local_rank)

    def dev_step():
        g = step(fact_dev, dim_dev, True, time_kernel=True)
        assert g == GROUPS, g
        torch.cuda.synchronize()
        kernel_ms.append(kev[0].elapsed_time(kev[1]))
        combine_partials()

    for _ in range(args.warmup):
        dev_step()
    kernel_ms.clear()
    clocks.start()
    ms_total, launches = timed(dev_step, args.steps, 0)
    clk = clocks.stop()
    ms_step = ms_total / args.steps
    value = world * n / (ms_step / 1e3)

    # ---- end to end from pinned host buffers ------------------------------
    e2e = None
    if args.e2e_steps > 0:
        h = [t.cpu().pin_memory() for t in (fk, qty, price, disc, key, grp)]
        fact_host = wg.Batch([wg.Column(I32, h[0].numpy()), wg.Column(I32, h[1].numpy()),
                              wg.Column(DEC, h[2].numpy().reshape(-1).view(wg.DEC_DTYPE), scale=2),
                              wg.Column(F64, h[3].numpy())])
        dim_host = wg.Batch([wg.Column(I32, h[4].numpy()), wg.Column(I32, h[5].numpy())])
        d2h = [0]

        def e2e_step():
            g = step(fact_host, dim_host, False)
            rows = agg.collect()
            d2h[0] = sum(v.nbytes + len(ok) for v, ok in rows)
            assert g == GROUPS
            combine_partials()

        e2e_ms, _ = timed(e2e_step, args.e2e_steps, 1)
        e2e = {"value": world * n / (e2e_ms / args.e2e_steps / 1e3), "unit": "rows/s",
               "h2d_bytes_per_step": n * FACT_BYTES_PER_ROW + DIM_ROWS * DIM_BYTES_PER_ROW,
               "d2h_bytes_per_step": d2h[0]}
        del h

    # ---- CPU baseline (rank 0, N = 1) ---------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rps, _ = cpu_pipeline_sample(CPU_SAMPLE_ROWS, threads, repeats=2)
        cpu = {"value": rps, "unit": "rows/s", "cores": threads, "kind": "port",
               "sample": f"{CPU_SAMPLE_ROWS} fact rows of the same workload (best of 2), C++ restatement of "
                         "the reference's Pipeline.Run with one worker per host thread"}

    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        k_ms = statistics.median(kernel_ms) if kernel_ms else None
        alg_bytes = n * FACT_BYTES_PER_ROW + DIM_ROWS * DIM_BYTES_PER_ROW + GROUPS * GROUP_STATE_BYTES
        achieved = alg_bytes / (k_ms / 1e3) / 1e9 if k_ms else None
        line = {
            "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int128+f64", "data": "synthetic",
            "config": {"workload": "star join + aggregate: 2^28 fact rows x 2^22 dim rows, qty>10, GROUP BY grp "
                                   "(1000 groups), SUM(price*(1-disc)) f64 + SUM(price) Int128",
                       "fact_rows_per_gpu": n, "dim_rows": DIM_ROWS, "groups": GROUPS,
                       "parallelism": f"dp{world}" if world > 1 else "single",
                       "l2": "inputs (8.6 GB/rank) larger than L2; no flush"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": None,
                         "kernel": "pipeline_kernel", "kernel_ms": k_ms, "algorithmic_bytes": alg_bytes,
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "gpu_launches_per_step": launches / args.steps,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    join.close()
    agg.close()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
