"""Benchmark of the B200 ksw_extend2 batch path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cfg2|cfg1|cfg4] [--schedule auto|plain|sorted|learned]

A step extends every job of one synthetic batch once: the uneven left+right extension
workload (about 1M jobs from 500k seeds on 100/150/250 bp reads, 20% unrelated targets,
w=100, BWA default scoring) unless --workload says otherwise.  `value` is GCUPS (useful DP
cells per second: the oracle's trip count of ksw.cu:346, summed over all jobs) with the
inputs resident in HBM; `e2e` is the same metric through the C ABI with host buffers, the
host->device copies of the job stream and the device->host copy of the results inside the
timed region.  With --gpus N each rank runs its own replica (the path has no exchange
step), so scaling is weak and `value` is the sum over ranks / the slowest rank's time.

--impl reference times the reference's own CPU ksw_extend2 (oracle/_ref, compiled from
bwa/src/ksw.cu) on all host threads over the same workload, or the C restatement of it
when oracle/_ref is absent.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ksw_extend2 GCUPS & extensions/s on 1 B200, learned vs plain schedule, bit-exact"
WORKLOADS = {
    # name: (synth kind, units, w, unrelated, description)
    "cfg2": (2, 500000, 100, 0.2,
             "uneven left+right ksw_extend2 batch: ~1M jobs from 500k seeds on 100/150/250 bp "
             "reads, divergence U[0,5%], 20% unrelated targets, w=100, a=1 b=4 o=6 e=1 zdrop=100"),
    "cfg1": (1, 100000, 100, 0.0,
             "100k right-extension jobs, qlen U[1,150], 1% subs / 0.1% indels, w=100 flank"),
    "cfg4": (4, 200000, 100, 0.0,
             "200k long-segment jobs, qlen log-uniform [500,5000], divergence U[0.1%,1%], w=100"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=sorted(WORKLOADS))
    ap.add_argument("--schedule", default="auto", choices=["auto", "plain", "sorted", "learned"])
    ap.add_argument("--seed", type=int, default=0x6A5 + 2)
    return ap.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi SM clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference(wl, threads):
    """Times the reference's own CPU ksw_extend2 (or the restatement) over the workload."""
    from tests import native as nat
    import g3sa_b200 as g
    sc = g.default_score()
    if nat.have_ref():
        kind = "reference"
        fn = lambda: nat.ref_extend(wl.jobs, wl.u8, sc, threads=threads)  # noqa: E731
    else:
        kind = "port"
        fn = lambda: nat.oracle_extend(wl.jobs, wl.u8, sc, threads=threads)[0]  # noqa: E731
    t0 = time.perf_counter()
    out = fn()
    dt = time.perf_counter() - t0
    return kind, dt, out


def useful_cells(wl):
    from tests import native as nat
    import g3sa_b200 as g
    _, cells, _ = nat.oracle_extend(wl.jobs, wl.u8, g.default_score(), threads=os.cpu_count() or 8)
    return int(cells.sum())


def run_reference_arm(args, ws, rank):
    import g3sa_b200 as g
    if rank != 0:
        return
    kind_, units, w, unrel, desc = WORKLOADS[args.workload]
    wl = g.synth(kind_, units, seed=args.seed, w=w, unrelated=unrel)
    threads = os.cpu_count() or 1
    cells = useful_cells(wl)
    times = []
    for it in range(args.warmup + args.steps):
        kind, dt, _ = cpu_reference(wl, threads)
        if it >= args.warmup:
            times.append(dt)
    t = sum(times) / len(times)
    gcups = cells / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gcups, 4), "unit": "GCUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
        "config": {"workload": desc, "jobs": wl.n, "cells": cells},
        "extensions_per_s": round(wl.n / t, 1),
        "cpu_baseline": {"value": round(gcups, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
                         "sample": f"whole workload ({wl.n} jobs) per step"},
        "e2e": {"value": round(gcups, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        return
    import torch
    import g3sa_b200 as g
    from g3sa_b200 import build
    build.build_lib()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    kind_, units, w, unrel, desc = WORKLOADS[args.workload]
    wl = g.synth(kind_, units, seed=args.seed + 1000 * rank, w=w, unrelated=unrel)
    codes, nmask = wl.planes()
    sc = g.default_score()
    n = wl.n
    mq, mt = int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max())
    ctx = g.Context(local)
    dev = torch.device("cuda", local)
    h_jobs = torch.from_numpy(wl.jobs.view(np.uint8).copy()).pin_memory()
    h_codes = torch.from_numpy(codes.view(np.uint8).copy()).pin_memory()
    h_nmask = torch.from_numpy(nmask.view(np.uint8).copy()).pin_memory()
    d_jobs = h_jobs.to(dev)
    d_codes = h_codes.to(dev)
    d_nmask = h_nmask.to(dev)
    d_out = torch.zeros((n, 6), dtype=torch.int32, device=dev)
    d_status = torch.zeros(n, dtype=torch.int32, device=dev)
    d_cells = torch.zeros(n, dtype=torch.int32, device=dev)
    h_out = torch.zeros((n, 6), dtype=torch.int32).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    sched = {"plain": g.SCHED_PLAIN, "sorted": g.SCHED_SORTED, "learned": g.SCHED_LEARNED,
             "auto": g.SCHED_SORTED}[args.schedule]
    lanes = 8

    def step(schedule, lanes_):
        ctx.extend_batch(sc, d_jobs, n, d_codes, d_nmask, d_out, d_status, mq, mt,
                         schedule=schedule, lanes=lanes_, d_cells=d_cells, stream=stream)

    # correctness gate and useful-cell count (device counter == oracle trip count)
    step(sched, lanes)
    torch.cuda.synchronize()
    st = d_status.cpu().numpy()
    if (st != 0).any():
        raise SystemExit(f"per-job status errors: {np.unique(st)}")
    cells = int(d_cells.to(torch.int64).sum().item())

    def timed(schedule, lanes_, k, w_):
        for _ in range(w_):
            step(schedule, lanes_)
        ms = []
        for _ in range(k):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(schedule, lanes_)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    ms = timed(sched, lanes, args.steps, args.warmup)
    barrier()
    clk = clocks.stop()
    t_step = sum(ms) / len(ms)

    # plain one-block-per-job kernel on the same batch, for the learned/plain comparison
    ms_plain = timed(g.SCHED_PLAIN, 0, max(2, args.steps // 2), 1)
    t_plain = sum(ms_plain) / len(ms_plain)

    # end to end through the C ABI with host buffers: H2D job stream, extension, D2H results
    bi = h_jobs.numel() + h_codes.numel() + h_nmask.numel()
    bo = h_out.numel() * 4

    def e2e_step():
        d_jobs.copy_(h_jobs, non_blocking=True)
        d_codes.copy_(h_codes, non_blocking=True)
        d_nmask.copy_(h_nmask, non_blocking=True)
        step(sched, lanes)
        h_out.copy_(d_out, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    barrier()
    t_e2e = sum(e2e_ms) / len(e2e_ms)

    # max over ranks, sums of work
    tot_cells, tot_jobs = cells, n
    if pg is not None:
        import torch.distributed as dist
        v = torch.tensor([t_step, t_e2e, t_plain], dtype=torch.float64, device=dev)
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
        t_step, t_e2e, t_plain = v.tolist()
        c = torch.tensor([tot_cells, tot_jobs], dtype=torch.int64, device=dev)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
        tot_cells, tot_jobs = c.tolist()

    peak_ops = ctx.int_peak()
    if rank == 0:
        gcups = tot_cells / (t_step * 1e-3) / 1e9
        peak_gcups = peak_ops / 8 / 1e9
        kind, cpu_t, _ = cpu_reference(wl, os.cpu_count() or 1)
        cpu_gcups = cells / cpu_t / 1e9
        line = {
            "metric": METRIC, "value": round(gcups, 3), "unit": "GCUPS", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator, shapes of the benchmark configuration)",
            "config": {"workload": desc, "jobs_per_gpu": n, "cells_per_gpu": cells,
                       "schedule": args.schedule, "lanes": lanes, "max_qlen": mq, "max_tlen": mt,
                       "l2": "256 MiB buffer written between timed steps", "parallelism": f"replicas x{ws}"},
            "extensions_per_s": round(tot_jobs / (t_step * 1e-3), 1),
            "plain": {"gcups": round(tot_cells / (t_plain * 1e-3) / 1e9, 3), "ms_per_step": round(t_plain, 4),
                      "schedule": "one 32-lane block per job, input order"},
            "speedup_vs_plain": round(t_plain / t_step, 3),
            "e2e": {"value": round(tot_cells / (t_e2e * 1e-3) / 1e9, 3), "unit": "GCUPS",
                    "ms_per_step": round(t_e2e, 4), "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo},
            "roofline": {"bound": "int_alu", "achieved": round(gcups / max(ws, 1), 3),
                         "peak": round(peak_gcups, 3), "unit": "GCUPS",
                         "frac": round(gcups / max(ws, 1) / peak_gcups, 4), "traffic": None,
                         "peak_source": "measured live: g3x_int_peak (DPX VIMNMX3 chains) / 8 ops per cell",
                         "int_ops_per_s": peak_ops},
            "cpu_baseline": {"value": round(cpu_gcups, 4), "unit": "GCUPS", "cores": os.cpu_count(),
                             "kind": kind, "sample": f"whole rank-0 workload ({n} jobs), one pass"},
            "clocks": clk,
            "gpu_launches": args.steps * 1,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
