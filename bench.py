"""Benchmark of the B200 ksw_extend2 batch path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cfg2|cfg1|cfg3|cfg4|cfg5|chains|global|seedsw] [--w W]
                    [--schedule auto|plain|sorted|learned]

A step extends every job of one synthetic batch once: the uneven left+right extension
workload (about 1M jobs from 500k seeds on 100/150/250 bp reads, 20% unrelated targets,
w=100, BWA default scoring) unless --workload says otherwise.  `value` is GCUPS (useful DP
cells per second: the oracle's trip count of ksw.cu:346, summed over all jobs) with the
inputs resident in HBM; `e2e` is the same metric through the C ABI with host buffers
(g3x_pipe): every step's host->device copies of the job stream and planes and device->host
copies of the results are inside the timed region, overlapped with the neighbouring steps'
extension.  With --gpus N each rank runs its own replica (the path has no exchange
step), so scaling is weak and `value` is the sum over ranks / the slowest rank's time.

--impl reference times the reference's own CPU ksw_extend2 (oracle/_ref, compiled from
bwa/src/ksw.cu) on all host threads over the same workload, or the C restatement of it
when oracle/_ref is absent.

`cfg3` is config 3's own recipe: the cost model trained on 2M traces of config 1's generator,
scheduling 1M held-out jobs of that generator (prediction error and warp idle fraction of
each schedule in the line).

`cfg5` is the seed-level band-retry stream (g3x_extend_seeds_stream, 2M seeds from host memory
in 64k-job chunks), learned width classes against the plain kernel, its regions compared with the
reference's own band-retry lines on the whole stream.

The other workloads measure the rows around the extension, each against the reference's own
CPU code for it: `chains` the chain-level call (g3x_chain2aln, mem_chain2aln over 60k reads),
`global` banded global alignment with backtrack (g3x_ksw_global2_batch, ksw_global2 over 200k
region pairs), `seedsw` the striped local alignment (g3x_ksw_align2_batch, ksw_align2 over
200k seed windows).
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
# DRAM bytes (read + write) per job staged by the int16x2 lane kernel, from the ncu capture of the
# width classes' launches summarised in profiles/lane16_kernel_cfg2_class_traffic.md
# (dram__bytes_read + dram__bytes_write of each class launch / its job count, 100k-seed case of the
# config-2 generator): a launch's DRAM traffic is its jobs' headers, query and target plane words
# and outputs, so it scales with the jobs the launch stages.  Keyed by the class's widest query.
TRAFFIC_PER_JOB = {32: 280.2, 56: 324.3, 88: 371.5, 128: 386.2, 168: 559.3, 200: 579.3, 232: 612.5}
WORKLOADS = {
    # name: (synth kind, units, w, unrelated, description with {w})
    "cfg2": (2, 500000, 100, 0.2,
             "uneven left+right ksw_extend2 batch: ~1M jobs from 500k seeds on 100/150/250 bp "
             "reads, divergence U[0,5%], 20% unrelated targets, w={w}, a=1 b=4 o=6 e=1 zdrop=100"),
    "cfg1": (1, 100000, 100, 0.0,
             "100k right-extension jobs, qlen U[1,150], 1% subs / 0.1% indels, w={w} flank"),
    "cfg3": (1, 1000000, 100, 0.0,
             "learned cost-model scheduling as config 3 states it: the model trained on 2M traces of "
             "config 1's generator, the schedule on 1M held-out jobs of that generator (right "
             "extensions, qlen U[1,150], 1% subs / 0.1% indels, w={w} flank)"),
    "cfg4": (4, 200000, 100, 0.0,
             "200k long-segment jobs, qlen log-uniform [500,5000], divergence U[0.1%,1%], indels "
             "up to 20 bp, w={w}, int32 scores (no int16 path)"),
}
# Trace units of the learned model's training batch per workload (the generator's units: seeds
# for cfg2, jobs otherwise), about 2M jobs where that stays within host memory.
TRAIN_UNITS = {"cfg2": 1_000_000, "cfg1": 2_000_000, "cfg3": 2_000_000, "cfg4": 200_000}


def workload(args):
    """(synth kind, units, w, unrelated fraction, description) of --workload with --w."""
    kind_, units, w, unrel, desc = WORKLOADS[args.workload]
    w = args.w if args.w else w
    return kind_, units, w, unrel, desc.format(w=w)


def bench_config(desc, n, cells):
    """The `config` object both arms print for one workload (the same keys and values)."""
    return {"workload": desc, "jobs": int(n), "cells": int(cells)}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=sorted(WORKLOADS) + ["cfg5", "chains", "global", "seedsw"])
    ap.add_argument("--schedule", default="auto", choices=["auto", "plain", "sorted", "learned"])
    ap.add_argument("--seed", type=int, default=0x6A5 + 2)
    ap.add_argument("--w", type=int, default=0, help="band width w of the job generator (0: the workload's)")
    return ap.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """SM clock / throttle-reason samples while the timed region runs: NVML read every 10 ms
    from a thread (reads only), or nvidia-smi at 200 ms where NVML cannot be loaded."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None
        self.nvml, self.samples, self.stop_flag = None, [], threading.Event()

    def _nvml_loop(self, nv, h):
        while not self.stop_flag.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception:   # noqa: BLE001 -- a failed read is a missing sample
                pass
            self.stop_flag.wait(0.01)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
            if len(vis) > self.gpu and vis[self.gpu].isdigit():         # the visible device's index
                h = nv.nvmlDeviceGetHandleByIndex(int(vis[self.gpu]))
            elif len(vis) > self.gpu and vis[self.gpu].startswith("GPU-"):
                h = nv.nvmlDeviceGetHandleByUUID(vis[self.gpu])
            else:
                h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self.nvml = nv
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
            return
        except Exception:   # noqa: BLE001 -- fall back to nvidia-smi
            self.nvml = None
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
        if self.nvml is not None:
            self.stop_flag.set()
            self.thread.join(timeout=2)
            nv, reasons = self.nvml, set()
            for _, _, bits in self.samples:
                for name, const in self.REASONS:
                    if bits & getattr(nv, const, 0):
                        reasons.add(name)
            sm = [c for c, _, _ in self.samples]
            try:
                nv.nvmlShutdown()
            except Exception:   # noqa: BLE001
                pass
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": max(m for _, m, _ in self.samples) if self.samples else None,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 10 ms"}
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
    kind_, units, w, unrel, desc = workload(args)
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
        "config": bench_config(desc, wl.n, cells),
        "extensions_per_s": round(wl.n / t, 1),
        "cpu_baseline": {"value": round(gcups, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
                         "sample": f"whole workload ({wl.n} jobs) per step"},
        "e2e": {"value": round(gcups, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


CHAIN_READS = 60000
CHAIN_DESC = ("mem_chain2aln over 60k synthetic reads (100/150/250 bp, divergence U[0,5%], small "
              "indels) on a 12-contig random reference: each read's true chain of exact-match seeds "
              "plus 0-2 spurious chains; seed order, containment skip, left/right extension with band "
              "retry, seed coverage; w=100, a=1 b=4 o=6 e=1 zdrop=100")


def ref_chains_threaded(wl, opt_cpu, threads):
    """The reference's own mem_chain2aln (oracle/_ref) over the reads, split into `threads`
    slices of reads run side by side (their regions go to disjoint seed slots)."""
    from concurrent.futures import ThreadPoolExecutor
    from g3sa_b200.chains import ALNREG_DT
    from tests import native as nat
    lib = nat.ref()
    ro = np.zeros(1, nat.REF_OPT_DT)
    for f in ("a", "o_del", "e_del", "o_ins", "e_ins", "pen_clip5", "pen_clip3", "w", "zdrop", "mat"):
        ro[f] = opt_cpu[f]
    u8 = np.ascontiguousarray(wl.u8)
    anns, chains, seeds = (np.ascontiguousarray(x) for x in (wl.anns, wl.chains, wl.seeds))
    regs = np.zeros(max(len(seeds), 1), ALNREG_DT)
    nregs = np.zeros(wl.n_reads, np.int32)
    bounds = np.linspace(0, wl.n_reads, threads + 1).astype(np.int64)

    def part(i):
        a, b = int(bounds[i]), int(bounds[i + 1])
        rd = np.ascontiguousarray(wl.reads[a:b])
        nr = np.zeros(b - a, np.int32)
        lib.g3r_chain2aln_reads(ro.ctypes.data, u8.ctypes.data, wl.ref_off, wl.l_pac, anns.ctypes.data,
                                len(anns), rd.ctypes.data, b - a, chains.ctypes.data, seeds.ctypes.data,
                                regs.ctypes.data, nr.ctypes.data)
        nregs[a:b] = nr

    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(part, range(threads)))
    return time.perf_counter() - t0, regs, nregs


def run_chain_workload(args, ws, rank):
    """`--workload chains`: the chain-level call (g3x_chain2aln), one step = every read of the
    batch; GCUPS from the oracle's DP cell count of the extensions the reads make."""
    import g3sa_b200 as g
    from g3sa_b200.chains import ALNREG_DT, synth_chains
    from tests import native as nat
    if args.impl == "reference" and rank != 0:
        return
    wl = synth_chains(CHAIN_READS, seed=args.seed + 1000 * rank)
    opt_cpu = nat.opt_from_score(g.default_score())
    oregs, onregs, ocells = nat.oracle_chains(wl, opt_cpu)
    cells = int(ocells.sum())
    threads = os.cpu_count() or 1
    metric = "mem_chain2aln GCUPS & reads/s on 1 B200, bit-exact"
    cfg = {"workload": CHAIN_DESC, "reads": wl.n_reads, "chains": len(wl.chains), "seeds": len(wl.seeds),
           "regions": int(onregs.sum()), "cells": cells}
    if args.impl == "reference":
        kind = "reference" if nat.have_ref() else "port"
        times = []
        for it in range(args.warmup + args.steps):
            if kind == "reference":
                dt, _, _ = ref_chains_threaded(wl, opt_cpu, threads)
            else:
                t0 = time.perf_counter()
                nat.oracle_chains(wl, opt_cpu)
                dt = time.perf_counter() - t0
            if it >= args.warmup:
                times.append(dt)
        t = sum(times) / len(times)
        gcups = cells / t / 1e9
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": round(gcups, 4), "unit": "GCUPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded)", "config": cfg, "reads_per_s": round(wl.n_reads / t, 1),
            "cpu_baseline": {"value": round(gcups, 4), "unit": "GCUPS", "cores": threads if kind == "reference" else 1,
                             "kind": kind, "sample": "whole workload per step"},
            "e2e": {"value": round(gcups, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return
    import torch
    from g3sa_b200 import build
    build.build_lib()
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    codes, nmask = wl.planes()
    host = {k: torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).copy()).pin_memory()
            for k, v in (("reads", wl.reads), ("chains", wl.chains), ("seeds", wl.seeds),
                         ("anns", wl.anns), ("codes", codes), ("nmask", nmask))}
    d = {k: v.to(dev) for k, v in host.items()}
    n_seeds = len(wl.seeds)
    d_regs = torch.zeros(n_seeds * ALNREG_DT.itemsize, dtype=torch.uint8, device=dev)
    d_nregs = torch.zeros(wl.n_reads, dtype=torch.int32, device=dev)
    d_status = torch.zeros(wl.n_reads, dtype=torch.int32, device=dev)
    h_regs = torch.zeros_like(d_regs, device="cpu").pin_memory()
    h_nregs = torch.zeros_like(d_nregs, device="cpu").pin_memory()
    h_status = torch.zeros_like(d_status, device="cpu").pin_memory()
    ctx = g.Context(local)
    # width classes of int16x2 lane kernels up to the longest read, the row-parallel kernel last
    tiles = [(16, 1, 4, 0, 32)] + [(wd, 1, 2, 0, 32) for wd in (32, 56, 88, 128, 176, 256)] + [(1 << 30, 32, 9, 0, 1)]
    ctx.set_tiles(tiles)
    opt = g.default_opt()
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def call(src):
        ctx.chain2aln(opt, wl.l_pac, wl.ref_off, src["anns"], len(wl.anns), src["reads"], wl.n_reads,
                      src["chains"], len(wl.chains), src["seeds"], n_seeds, src["codes"], src["nmask"],
                      d_regs, d_nregs, d_status, schedule=g.SCHED_SORTED, stream=stream)

    call(d)
    torch.cuda.synchronize()
    regs = d_regs.cpu().numpy().view(ALNREG_DT)
    nregs = d_nregs.cpu().numpy()
    exact = bool((d_status == 0).all()) and np.array_equal(nregs, onregs) and np.array_equal(
        nat.region_rows(regs, nregs, wl.chains, wl.reads), nat.region_rows(oregs, onregs, wl.chains, wl.reads))
    if not exact:
        raise SystemExit("chain-level results differ from the oracle")
    clocks = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    clocks.start()
    ms = timed_steps(lambda: call(d), args.steps, args.warmup, stream, flush)
    clk = clocks.stop()

    def e2e_step():
        for k in d:
            d[k].copy_(host[k], non_blocking=True)
        call(d)
        h_regs.copy_(d_regs, non_blocking=True)
        h_nregs.copy_(d_nregs, non_blocking=True)
        h_status.copy_(d_status, non_blocking=True)

    e2e_ms = timed_steps(e2e_step, max(3, args.steps // 4), args.warmup, stream, flush)
    t = sum(ms) / len(ms)
    te = sum(e2e_ms) / len(e2e_ms)
    (t, te), (tot_cells, tot_reads) = combine_ranks(dist, [t, te], [cells, wl.n_reads], dev)
    if rank != 0:
        return
    peak_gcups = ctx.int_peak() / 8 / 1e9
    cpu_t, _, _ = ref_chains_threaded(wl, opt_cpu, threads) if nat.have_ref() else (None, None, None)
    gcups = tot_cells / (t * 1e-3) / 1e9
    bi = sum(v.numel() for v in host.values())
    bo = h_regs.numel() + 4 * (h_nregs.numel() + h_status.numel())
    print(json.dumps({
        "metric": metric, "value": round(gcups, 3), "unit": "GCUPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)", "config": cfg,
        "reads_per_s": round(tot_reads / (t * 1e-3), 1),
        "e2e": {"value": round(tot_cells / (te * 1e-3) / 1e9, 3), "unit": "GCUPS", "ms_per_step": round(te, 4),
                "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo},
        "roofline": {"bound": "int_alu", "achieved": round(gcups / max(ws, 1), 3), "peak": round(peak_gcups, 3),
                     "unit": "GCUPS", "frac": round(gcups / max(ws, 1) / peak_gcups, 4), "traffic": None,
                     "note": "the whole call (waves of seed-level extension through the width classes) "
                             "against the int-ALU cells/s peak"},
        "cpu_baseline": None if cpu_t is None else {
            "value": round(cells / cpu_t / 1e9, 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
            "sample": "whole rank-0 workload, one pass, the reference's own mem_chain2aln"},
        "clocks": clk, "outputs_equal_oracle": exact,
        # per step: prep, resolve and finish, the five seed-level passes and four extension
        # waves of (cost, scan, scatter, one launch per width class)
        "gpu_launches": args.steps * (3 + 5 + 4 * (3 + len(tiles))), "width_classes": tiles,
    }), flush=True)


CFG5_SEEDS = 2_000_000
CFG5_CHUNK = 32768       # seeds per chunk: 64k extension jobs, a left and a right one per seed
CFG5_DESC = ("band-retry stream: 2M seeds of the uneven left+right generator (100/150/250 bp reads, divergence "
             "U[0,5%], 20% unrelated targets) = 4M ksw_extend2 jobs before retries, each side run with w=100 "
             "and again with w=200 when the score changed and max_off >= 3w/4 (at most 2 tries), from pinned "
             "host memory in 64k-job chunks (32k seeds), pinned copies with seven chunks in flight (the config's "
             "double buffering, two sets deeper); a=1 b=4 o=6 e=1 zdrop=100")


def seeds_threaded(fn, seeds, u8, opt, threads):
    """fn (the oracle's or the reference's seed driver) over `threads` slices of the seeds run side
    by side (the ctypes calls release the interpreter lock); returns the concatenated records."""
    from concurrent.futures import ThreadPoolExecutor
    bounds = np.linspace(0, len(seeds), threads + 1).astype(np.int64)
    parts = [np.ascontiguousarray(seeds[bounds[i]:bounds[i + 1]]) for i in range(threads)]
    with ThreadPoolExecutor(threads) as ex:
        outs = list(ex.map(lambda p: fn(p, u8, opt), parts))
    return np.concatenate(outs)


def run_cfg5_workload(args, ws, rank):
    """`--workload cfg5`: the seed-level band-retry stream (g3x_extend_seeds_stream) over 2M seeds
    in 64k-job chunks, the learned width-class schedule against the plain kernel; the regions
    are compared with the reference's own band-retry lines on the whole stream."""
    import g3sa_b200 as g
    from tests import native as nat
    if args.impl == "reference" and rank != 0:
        return
    wl = g.synth(2, CFG5_SEEDS, seed=args.seed + 1000 * rank, w=100, unrelated=0.2)
    sc = g.default_score()
    opt_cpu = nat.opt_from_score(sc, w=100)
    threads = os.cpu_count() or 1
    oreg = seeds_threaded(nat.oracle_seeds, wl.seeds, wl.u8, opt_cpu, threads)
    cells = int(oreg["cells"].sum())
    n = len(wl.seeds)
    cfg = bench_config(CFG5_DESC, n, cells)
    kind = "reference" if nat.have_ref() else "port"
    cpu_fn = nat.ref_seeds if kind == "reference" else nat.oracle_seeds
    if args.impl == "reference":
        times = []
        for it in range(args.warmup + min(args.steps, 3)):
            t0 = time.perf_counter()
            seeds_threaded(cpu_fn, wl.seeds, wl.u8, opt_cpu, threads)
            if it >= args.warmup:
                times.append(time.perf_counter() - t0)
        t = sum(times) / len(times)
        gcups = cells / t / 1e9
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": round(gcups, 4), "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)", "config": cfg,
            "seeds_per_s": round(n / t, 1),
            "cpu_baseline": {"value": round(gcups, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
                             "sample": "whole workload per step (the reference's band-retry lines, threads over seed slices)"},
            "e2e": {"value": round(gcups, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return
    import torch
    from g3sa_b200 import build, learn
    build.build_lib()
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    codes, nmask = wl.planes()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).pin_memory()  # noqa: E731
    h_seeds, h_codes, h_nmask = pin(g.device_seeds(wl.seeds)), pin(codes), pin(nmask)
    h_regs = torch.zeros(n * g.REG_DT.itemsize, dtype=torch.uint8).pin_memory()
    h_status = torch.full((n,), 99, dtype=torch.int32).pin_memory()
    mq = int(wl.seeds["l_query"].max())
    mt = int((wl.seeds["rmax1"] - wl.seeds["rmax0"]).max())
    ctx = g.Context(local)
    # the cost model on traces of a held-out job batch of the generator, and width classes tuned
    # for the learned order on another such batch
    train_metrics = learn.train(ctx, n_train=TRAIN_UNITS["cfg2"], seed_train=0xA11CE + rank, kind=2, w=100,
                                unrelated=0.2)
    tw = g.synth(2, 200000, seed=args.seed + 7 + 1000 * rank, w=100, unrelated=0.2)
    tc, tn = tw.planes()
    td = [torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).copy()).to(dev) for x in (tw.jobs, tc, tn)]
    tiles = ctx.autotune(sc, td[0], tw.n, td[1], td[2], int(tw.jobs["qlen"].max()), int(tw.jobs["tlen"].max()),
                         schedule=g.SCHED_LEARNED)
    del td
    opt = g.default_opt(w=100)
    stream = torch.cuda.current_stream(dev)

    def call(sched):
        ctx.extend_seeds_stream(opt, h_seeds, h_codes, h_nmask, len(wl.u8), h_regs, h_status, mq, mt,
                                chunk=CFG5_CHUNK, schedule=sched)

    # the region fields mem_chain2aln sets; the try counts are the library's and the oracle's own
    fields = ("rb", "re", "qb", "qe", "score", "truesc", "w")
    regs = {}
    for name, sched in (("plain", g.SCHED_PLAIN), ("learned", g.SCHED_LEARNED)):
        h_status.fill_(99)
        call(sched)
        if (h_status.numpy() != 0).any():
            raise SystemExit(f"{name}: seed errors in the stream")
        regs[name] = h_regs.numpy().view(g.REG_DT).copy()
    t0 = time.perf_counter()
    ref_reg = seeds_threaded(cpu_fn, wl.seeds, wl.u8, opt_cpu, threads) if rank == 0 else None
    cpu_t = time.perf_counter() - t0
    same_plain = all(np.array_equal(regs["plain"][f], regs["learned"][f]) for f in fields + ("tries_left", "tries_right"))
    same_plain = same_plain and all(np.array_equal(regs["learned"][f], oreg[f]) for f in ("tries_left", "tries_right"))
    same_ref = ref_reg is None or all(np.array_equal(regs["learned"][f], ref_reg[f]) for f in fields)
    if not (same_plain and same_ref):
        raise SystemExit("stream regions differ between schedules or from the reference")

    def timed(sched, k, w):
        for _ in range(w):
            call(sched)
        ms = []
        for _ in range(k):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call(sched)          # blocks until every chunk's regions are back in host memory
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return sum(ms) / len(ms)

    clocks = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    clocks.start()
    t_learned = timed(g.SCHED_LEARNED, args.steps, args.warmup)
    clk = clocks.stop()
    k2 = max(2, args.steps // 2)
    t_plain = timed(g.SCHED_PLAIN, k2, 1)
    t_sorted = timed(g.SCHED_SORTED, k2, 1)
    (t_learned, t_plain, t_sorted), (tot_cells, tot_n) = combine_ranks(dist, [t_learned, t_plain, t_sorted],
                                                                       [cells, n], dev)
    if rank != 0:
        return
    gcups = tot_cells / (t_learned * 1e-3) / 1e9
    peak16 = 2 * ctx.int_peak() / 8 / 1e9
    bi = h_seeds.numel() + h_codes.numel() + h_nmask.numel()
    bo = h_regs.numel() + 4 * h_status.numel()
    gc = lambda t: round(tot_cells / (t * 1e-3) / 1e9, 3)  # noqa: E731
    chunks = (n + CFG5_CHUNK - 1) // CFG5_CHUNK
    print(json.dumps({
        "metric": METRIC, "value": round(gcups, 3), "unit": "GCUPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_learned, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int16x2 (int32 where the fit fails)", "data": "synthetic (seeded generator)",
        "config": cfg,
        "setup": {"chunk_seeds": CFG5_CHUNK, "chunks": chunks, "width_classes": tiles,
                  "note": "the workload lives in host memory: every step copies each chunk's seeds and plane "
                          "words in and its regions out (pinned staging, seven chunks in flight); value and e2e are the same "
                          "measurement"},
        "seeds_per_s": round(tot_n / (t_learned * 1e-3), 1),
        "extensions_per_s": round(int(regs["learned"]["tries_left"].sum() + regs["learned"]["tries_right"].sum())
                                  / (t_learned * 1e-3), 1),
        "arms": {"learned": {"gcups": gc(t_learned), "ms": round(t_learned, 4)},
                 "sorted": {"gcups": gc(t_sorted), "ms": round(t_sorted, 4)},
                 "plain": {"gcups": gc(t_plain), "ms": round(t_plain, 4),
                           "kernel": "one 32-lane block per job, anti-diagonal wavefront"}},
        "speedup_learned_vs_plain": round(t_plain / t_learned, 3),
        "speedup_learned_vs_sorted": round(t_sorted / t_learned, 3),
        "cost_model": train_metrics,
        "e2e": {"value": round(gcups, 3), "unit": "GCUPS", "ms_per_step": round(t_learned, 4),
                "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                "api": "g3x_extend_seeds_stream per step (pinned host seeds, planes and regions)"},
        "roofline": {"bound": "int_alu", "achieved": round(gcups / max(ws, 1), 3), "peak": round(peak16, 3),
                     "unit": "GCUPS", "frac": round(gcups / max(ws, 1) / peak16, 4), "traffic": None,
                     "note": "the whole stream (copies, seed waves, band retries) against the int16x2 cells/s "
                             "roofline (measured 32-bit int ops/s / 8 ops per cell x 2)"},
        "cpu_baseline": {"value": round(cells / cpu_t / 1e9, 4), "unit": "GCUPS", "cores": threads, "kind": kind,
                         "sample": "whole rank-0 workload, one pass: the reference's band-retry lines, threads over seed slices",
                         "gpu_regions_identical": same_ref},
        "clocks": clk, "outputs_equal_plain_kernel": same_plain,
        # per chunk: the seed rebase, the five seed-level passes and four extension waves of
        # (learned keys, scan, scatter, one launch per width class)
        "gpu_launches": args.steps * -(-n // CFG5_CHUNK) * (1 + 5 + 4 * (3 + len(tiles))),
    }), flush=True)


# DRAM bytes (read + write) per launch of the dominant kernel of each workload below, from ncu
# captures of these workloads (global_kernel: 0.427 GB read + 1.010 GB written; sw_kernel<16>:
# 18.9 MB read, nothing written back but the outputs)
GLOBAL_DRAM_BYTES = 1_436_724_000
SW_DRAM_BYTES = 18_913_024
GLOBAL_JOBS = 200000
GLOBAL_DESC = ("ksw_global2 with backtrack over 200k synthetic region pairs as the traceback stage issues "
               "them: query U[0,250) bases, target = query with up to 5 substitutions/1-base indels, 10% "
               "with N codes, band w in {5, 10, 20, 50}; a=1 b=4 o=6 e=1")


def run_global_workload(args, ws, rank):
    """`--workload global`: g3x_ksw_global2_batch, one step = every job of the batch once;
    GCUPS from the oracle's DP cell count."""
    import g3sa_b200 as g
    from concurrent.futures import ThreadPoolExecutor
    from tests import native as nat
    if args.impl == "reference" and rank != 0:
        return
    cj, u8 = nat.global_jobs(GLOBAL_JOBS, args.seed + 1000 * rank, max_len=250, ws=(5, 10, 20, 50))
    n = len(cj)
    stride = int((cj["qlen"] + cj["tlen"]).max()) + 2
    sc = g.default_score()
    s_o, c_o, n_o, cells_o = nat.oracle_global(cj, u8, sc, stride)
    cells = int(cells_o.sum())
    # the GPU's CIGAR slots hold the longest CIGAR of the batch (a caller sizes them likewise)
    gstride = int(n_o.max()) + 2
    threads = os.cpu_count() or 1
    metric = "ksw_global2 GCUPS & alignments/s on 1 B200, bit-exact"
    cfg = {"workload": GLOBAL_DESC, "jobs": n, "cells": cells, "cigar_slots": int(n_o.max()) + 2}

    def ref_time():
        bounds = np.linspace(0, n, threads + 1).astype(np.int64)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda i: nat.ref_global(cj[bounds[i]:bounds[i + 1]], u8, sc, stride), range(threads)))
        return time.perf_counter() - t0

    if args.impl == "reference":
        kind = "reference" if nat.have_ref() else "port"
        times = []
        for it in range(args.warmup + args.steps):
            if kind == "reference":
                dt = ref_time()
            else:
                t0 = time.perf_counter()
                nat.oracle_global(cj, u8, sc, stride)
                dt = time.perf_counter() - t0
            if it >= args.warmup:
                times.append(dt)
        t = sum(times) / len(times)
        gcups = cells / t / 1e9
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": round(gcups, 4), "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)", "config": cfg,
            "alignments_per_s": round(n / t, 1),
            "cpu_baseline": {"value": round(gcups, 4), "unit": "GCUPS", "cores": threads if kind == "reference" else 1,
                             "kind": kind, "sample": "whole workload per step"},
            "e2e": {"value": round(gcups, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return
    import torch
    from g3sa_b200 import build
    build.build_lib()
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    jobs = np.zeros(n, g.JOB_DT)
    jobs["q_off"], jobs["t_off"] = cj["q_off"], cj["t_off"]
    jobs["qlen"], jobs["tlen"], jobs["w"] = cj["qlen"], cj["tlen"], cj["w"]
    codes, nmask = g.pack_planes(u8)
    host = {k: torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).copy()).pin_memory()
            for k, v in (("jobs", jobs), ("codes", codes), ("nmask", nmask))}
    d = {k: v.to(dev) for k, v in host.items()}
    d_score = torch.zeros(n, dtype=torch.int32, device=dev)
    d_cig = torch.zeros(n * gstride, dtype=torch.int32, device=dev)
    d_nc = torch.zeros(n, dtype=torch.int32, device=dev)
    d_st = torch.zeros(n, dtype=torch.int32, device=dev)
    ctx = g.Context(local)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    mq, mt, mw = int(cj["qlen"].max()), int(cj["tlen"].max()), int(cj["w"].max())

    def call():
        ctx.global_batch(sc, d["jobs"], n, d["codes"], d["nmask"], mq, mt, mw, d_score, d_cig, gstride, d_nc, d_st,
                         stream=stream)

    call()
    torch.cuda.synchronize()
    cig = d_cig.cpu().numpy().view(np.uint32).reshape(n, gstride)
    nc = d_nc.cpu().numpy()
    exact = bool((d_st == 0).all()) and np.array_equal(d_score.cpu().numpy(), s_o) and np.array_equal(nc, n_o) and \
        all(np.array_equal(cig[k, :nc[k]], c_o[k, :n_o[k]]) for k in range(n))
    if not exact:
        raise SystemExit("global alignments differ from the oracle")
    clocks = ClockSampler(local)
    clocks.start()
    ms = timed_steps(call, args.steps, args.warmup, stream, flush)
    clk = clocks.stop()

    # end to end: two contexts, streams and buffer sets, so one batch's copies overlap the
    # other's alignment
    def run_g(cx, dd, outs, st):
        cx.global_batch(sc, dd["jobs"], n, dd["codes"], dd["nmask"], mq, mt, mw, outs[0], outs[1], gstride,
                        outs[2], outs[3], stream=st)

    submit, wait, sets = two_set_pipeline(lambda i: ctx if i == 0 else g.Context(local), host,
                                          (d_score, d_cig, d_nc, d_st), run_g)
    te = timed_pipeline(submit, wait, max(3, args.steps // 4), args.warmup, stream, flush)
    torch.cuda.synchronize()
    for st_, dd, outs, h_outs, cx in sets:     # both sets' last batches came back intact
        exact = exact and np.array_equal(h_outs[0].numpy(), s_o) and bool((h_outs[3] == 0).all())
    t = sum(ms) / len(ms)
    (t, te), (tot_cells, tot_n) = combine_ranks(dist, [t, te], [cells, n], dev)
    if rank != 0:
        return
    peak_gcups = ctx.int_peak() / 8 / 1e9
    cpu_t = ref_time() if nat.have_ref() else None
    gcups = tot_cells / (t * 1e-3) / 1e9
    bi = sum(v.numel() for v in host.values())
    bo = sum(h.numel() * h.element_size() for h in sets[0][3])
    print(json.dumps({
        "metric": metric, "value": round(gcups, 3), "unit": "GCUPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)", "config": cfg,
        "alignments_per_s": round(tot_n / (t * 1e-3), 1),
        "e2e": {"value": round(tot_cells / (te * 1e-3) / 1e9, 3), "unit": "GCUPS", "ms_per_step": round(te, 4),
                "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                "overlap": "two contexts, streams and buffer sets: a batch's copies overlap the other set's batch"},
        "roofline": {"bound": "int_alu", "achieved": round(gcups / max(ws, 1), 3), "peak": round(peak_gcups, 3),
                     "unit": "GCUPS", "frac": round(gcups / max(ws, 1) / peak_gcups, 4),
                     "traffic": GLOBAL_DRAM_BYTES,
                     "note": "cells per second of the global kernel against the int-ALU cells/s peak (8 ops per cell); "
                             "traffic: DRAM bytes read + written by one global_kernel launch of this workload "
                             "(an ncu capture of it): the direction bytes"},
        "cpu_baseline": None if cpu_t is None else {
            "value": round(cells / cpu_t / 1e9, 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
            "sample": "whole rank-0 workload, one pass, the reference's own ksw_global2"},
        "clocks": clk, "outputs_equal_oracle": exact, "gpu_launches": args.steps,
    }), flush=True)


SW_JOBS = 200000
SW_DESC = ("ksw_align2 (16-bit striped local SW, KSW_XSTART as mem_seed_sw calls it) over 200k synthetic "
           "seed windows as mem_seed_sw cuts them: seed U[19,60) bases with U[0,50] bases either side on the "
           "read and the reference, half the flanks related (divergence U[0,10%]), half unrelated, core 2%, "
           "5% of queries with N codes; a=1 b=4 o=6 e=1")


def run_sw_workload(args, ws, rank):
    """`--workload seedsw`: g3x_ksw_align2_batch with KSW_XSTART, one step = every window of the
    batch once (forward pass and start-position pass); GCUPS from the oracle's cell count
    (query length x target rows entered, both passes)."""
    import g3sa_b200 as g
    from concurrent.futures import ThreadPoolExecutor
    from tests import native as nat
    if args.impl == "reference" and rank != 0:
        return
    cj, u8 = nat.sw_windows(SW_JOBS, args.seed + 2000 + 1000 * rank)
    n = len(cj)
    sc = g.default_score()
    xtra = g.KSW_XSTART
    want, cells_o = nat.oracle_sw(cj, u8, sc, xtra)
    cells = int(cells_o.sum())
    threads = os.cpu_count() or 1
    metric = "ksw_align2 GCUPS & alignments/s on 1 B200, bit-exact"
    cfg = {"workload": SW_DESC, "jobs": n, "cells": cells, "xtra": "KSW_XSTART"}

    def ref_time():
        bounds = np.linspace(0, n, threads + 1).astype(np.int64)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda i: nat.ref_sw(cj[bounds[i]:bounds[i + 1]], u8, sc, xtra), range(threads)))
        return time.perf_counter() - t0

    if args.impl == "reference":
        kind = "reference" if nat.have_ref() else "port"
        times = []
        for it in range(args.warmup + args.steps):
            if kind == "reference":
                dt = ref_time()
            else:
                t0 = time.perf_counter()
                nat.oracle_sw(cj, u8, sc, xtra)
                dt = time.perf_counter() - t0
            if it >= args.warmup:
                times.append(dt)
        t = sum(times) / len(times)
        gcups = cells / t / 1e9
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": round(gcups, 4), "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16x2", "data": "synthetic (seeded)", "config": cfg,
            "alignments_per_s": round(n / t, 1),
            "cpu_baseline": {"value": round(gcups, 4), "unit": "GCUPS", "cores": threads if kind == "reference" else 1,
                             "kind": kind, "sample": "whole workload per step"},
            "e2e": {"value": round(gcups, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return
    import torch
    from g3sa_b200 import build
    build.build_lib()
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    jobs = np.zeros(n, g.JOB_DT)
    for f in ("q_off", "t_off", "qlen", "tlen", "flags"):
        jobs[f] = cj[f]
    codes, nmask = g.pack_planes(u8)
    host = {k: torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).copy()).pin_memory()
            for k, v in (("jobs", jobs), ("codes", codes), ("nmask", nmask))}
    d = {k: v.to(dev) for k, v in host.items()}
    d_out = torch.zeros(n * 7, dtype=torch.int32, device=dev)
    d_st = torch.zeros(n, dtype=torch.int32, device=dev)
    ctx = g.Context(local)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    mt = int(cj["tlen"].max())

    def call():
        ctx.align2_batch(sc, d["jobs"], n, d["codes"], d["nmask"], xtra, mt, d_out, d_st, stream=stream)

    call()
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().view(g.SWR_DT)
    exact = bool((d_st == 0).all()) and np.array_equal(got, want)
    if not exact:
        raise SystemExit("local alignments differ from the oracle")
    clocks = ClockSampler(local)
    clocks.start()
    ms = timed_steps(call, args.steps, args.warmup, stream, flush)
    clk = clocks.stop()

    def run_s(cx, dd, outs, st):
        cx.align2_batch(sc, dd["jobs"], n, dd["codes"], dd["nmask"], xtra, mt, outs[0], outs[1], stream=st)

    submit, wait, sets = two_set_pipeline(lambda i: ctx if i == 0 else g.Context(local), host, (d_out, d_st), run_s)
    te = timed_pipeline(submit, wait, max(3, args.steps // 4), args.warmup, stream, flush)
    torch.cuda.synchronize()
    for st_, dd, outs, h_outs, cx in sets:     # both sets' last batches came back intact
        exact = exact and np.array_equal(h_outs[0].numpy().view(g.SWR_DT), want) and bool((h_outs[1] == 0).all())
    t = sum(ms) / len(ms)
    (t, te), (tot_cells, tot_n) = combine_ranks(dist, [t, te], [cells, n], dev)
    if rank != 0:
        return
    peak_gcups = ctx.int_peak() / 8 / 1e9
    cpu_t = ref_time() if nat.have_ref() else None
    gcups = tot_cells / (t * 1e-3) / 1e9
    bi = sum(v.numel() for v in host.values())
    bo = sum(h.numel() * h.element_size() for h in sets[0][3])
    print(json.dumps({
        "metric": metric, "value": round(gcups, 3), "unit": "GCUPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int16x2", "data": "synthetic (seeded generator)", "config": cfg,
        "alignments_per_s": round(tot_n / (t * 1e-3), 1),
        "e2e": {"value": round(tot_cells / (te * 1e-3) / 1e9, 3), "unit": "GCUPS", "ms_per_step": round(te, 4),
                "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                "overlap": "two contexts, streams and buffer sets: a batch's copies overlap the other set's batch"},
        "roofline": {"bound": "int_alu", "achieved": round(gcups / max(ws, 1), 3), "peak": round(peak_gcups, 3),
                     "unit": "GCUPS", "frac": round(gcups / max(ws, 1) / peak_gcups, 4),
                     "traffic": SW_DRAM_BYTES,
                     "note": "cells per second of the step against the int-ALU cells/s peak (8 ops per cell); "
                             "traffic: DRAM bytes of one sw_kernel<16> launch (the class with 83% of the cells) of "
                             "this workload (an ncu capture of it): job headers and planes"},
        "cpu_baseline": None if cpu_t is None else {
            "value": round(cells / cpu_t / 1e9, 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
            "sample": "whole rank-0 workload, one pass, the reference's own ksw_align2 (trap line left out)"},
        "clocks": clk, "outputs_equal_oracle": exact, "gpu_launches": 6 * args.steps,
    }), flush=True)


def two_set_pipeline(make_ctx, host, outs_like, run):
    """A caller's pipeline over the public API: batches alternate between two contexts, each
    with its own stream and device buffer set; batch k's host->device copies (pinned), its
    call `run(ctx, d, outs, stream)` and its device->host copies are enqueued on its set's
    stream, so they overlap the other set's batch.  Returns (submit, wait, sets) for
    timed_pipeline; each set is (stream, d, outs, h_outs)."""
    import torch
    sets = []
    for i in range(2):
        st = torch.cuda.Stream()
        d = {k: torch.empty(v.shape, dtype=v.dtype, device="cuda") for k, v in host.items()}
        outs = [torch.empty_like(x) for x in outs_like]
        h_outs = [torch.empty(x.shape, dtype=x.dtype).pin_memory() for x in outs]
        sets.append((st, d, outs, h_outs, make_ctx(i)))
    k = [0]

    def submit():
        st, d, outs, h_outs, cx = sets[k[0] % 2]
        k[0] += 1
        st.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(st):
            for name in d:
                d[name].copy_(host[name], non_blocking=True)
            run(cx, d, outs, st)
            for h, x in zip(h_outs, outs):
                h.copy_(x, non_blocking=True)

    def wait(stream):
        for st in sets:
            stream.wait_stream(st[0])

    return submit, wait, sets


def combine_ranks(dist, times, counts, device):
    """Every rank calls this with its own step times and counts: returns the max over ranks
    of each time (the slowest replica sets the pace) and the sum over ranks of each count.
    Without a process group it returns the inputs."""
    import torch
    if dist is None:
        return list(times), list(counts)
    v = torch.tensor(list(times), dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.MAX)
    c = torch.tensor(list(counts), dtype=torch.int64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return v.tolist(), c.tolist()


def timed_steps(fn, k, w, stream, flush, nvtx=None):
    """W untimed calls, then K calls each bracketed by CUDA events on `stream`, with a
    256 MiB write between them so no step starts with the previous step's data in L2.  With
    `nvtx`, the K timed calls sit inside an NVTX range of that name (for profiler filters)."""
    import torch
    for _ in range(w):
        fn()
    ms = []
    if nvtx:
        torch.cuda.nvtx.range_push(nvtx)
    for _ in range(k):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    if nvtx:
        torch.cuda.nvtx.range_pop()
    return ms


def kernel_name(t):
    """Kernel of a width class (width, lanes, tile, warp_batch, refill)."""
    if t[1] != 1:
        return f"band {t[2]}" if t[2] >= 64 else f"rowpar g{t[1]} c{t[2]}"
    if t[2] >= 64:
        return f"lane ring {t[2]}"
    return {2: "lane16", 4: "lane2"}.get(t[2], "lane")


def timed_pipeline(submit, wait, k, w, stream, flush):
    """W untimed submits, then K submits between two CUDA events on `stream`, the second
    recorded after `wait(stream)` (the K batches' outputs are on the host); the 256 MiB write
    precedes every submit.  Returns ms per step."""
    import torch
    for _ in range(w):
        flush.fill_(1)
        submit()
    wait(stream)
    stream.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        flush.fill_(1)
        submit()
    wait(stream)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / k


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.workload == "chains":
        run_chain_workload(args, ws, rank)
        return
    if args.workload == "global":
        run_global_workload(args, ws, rank)
        return
    if args.workload == "seedsw":
        run_sw_workload(args, ws, rank)
        return
    if args.workload == "cfg5":
        run_cfg5_workload(args, ws, rank)
        return
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        return
    import torch
    import g3sa_b200 as g
    from g3sa_b200 import build, learn
    build.build_lib()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    kind_, units, w, unrel, desc = workload(args)
    wl = g.synth(kind_, units, seed=args.seed + 1000 * rank, w=w, unrelated=unrel)
    codes, nmask = wl.planes()
    sc = g.default_score()
    n = wl.n
    mq, mt = int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max())
    ctx = g.Context(local)
    if args.workload == "cfg4":
        ctx.set_int16(False)    # long segments are scored in int32: no int16x2 class
    dev = torch.device("cuda", local)
    h_jobs = torch.from_numpy(wl.jobs.view(np.uint8).copy()).pin_memory()
    h_codes = torch.from_numpy(codes.view(np.uint8).copy()).pin_memory()
    h_nmask = torch.from_numpy(nmask.view(np.uint8).copy()).pin_memory()
    d_jobs, d_codes, d_nmask = h_jobs.to(dev), h_codes.to(dev), h_nmask.to(dev)
    d_out = torch.zeros((n, 6), dtype=torch.int32, device=dev)
    d_status = torch.zeros(n, dtype=torch.int32, device=dev)
    d_cells = torch.zeros(n, dtype=torch.int32, device=dev)
    d_rows = torch.zeros(n, dtype=torch.int32, device=dev)
    h_out = torch.zeros((n, 6), dtype=torch.int32).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    def batch(schedule, **kw):
        ctx.extend_batch(sc, d_jobs, n, d_codes, d_nmask, d_out, d_status, mq, mt,
                         schedule=schedule, stream=stream, **kw)

    # Useful cells of this batch: the kernels' own trip-count counters (plain kernel).
    batch(g.SCHED_PLAIN, d_cells=d_cells, d_rows=d_rows)
    torch.cuda.synchronize()
    if (d_status != 0).any():
        raise SystemExit("per-job status errors in the plain run")
    cells_np = d_cells.cpu().numpy()
    cells = int(cells_np.astype(np.int64).sum())
    plain_out = d_out.cpu().numpy().copy()

    # Learned cost model: trained on the GPU on plain-kernel traces of a held-out batch of the
    # same generator (another seed), about 2M jobs.
    train_metrics = learn.train(ctx, n_train=TRAIN_UNITS[args.workload],
                                seed_train=0xA11CE + rank, kind=kind_, w=w, unrelated=unrel)
    pred_err = learn.prediction_error(ctx, wl.jobs, d_jobs, n, d_codes, d_nmask, d_rows.cpu().numpy())

    # Autotune the width classes on this batch for each schedule's own job order, and capture
    # each schedule's graph with its own tiles (a graph keeps the launch configuration it was
    # captured with).
    t_tune = time.perf_counter()
    sched = {"plain": g.SCHED_PLAIN, "sorted": g.SCHED_SORTED, "learned": g.SCHED_LEARNED,
             "auto": g.SCHED_LEARNED}[args.schedule]
    graphs, tiles_of = {}, {}
    for sname, sval in (("sorted", g.SCHED_SORTED), ("learned", g.SCHED_LEARNED)):
        tiles_of[sname] = ctx.autotune(sc, d_jobs, n, d_codes, d_nmask, mq, mt, schedule=sval)
        graphs[sname] = ctx.capture_batch(sc, d_jobs, n, d_codes, d_nmask, d_out, d_status, mq, mt,
                                          schedule=sval)
    t_tune = time.perf_counter() - t_tune
    tiles = tiles_of["learned" if sched != g.SCHED_SORTED else "sorted"]
    ctx.set_tiles(tiles)
    main_graph = graphs["learned" if sched == g.SCHED_LEARNED else "sorted"]
    if sched == g.SCHED_PLAIN:
        main_fn = lambda: batch(g.SCHED_PLAIN)  # noqa: E731
    else:
        main_fn = lambda: main_graph.launch(stream)  # noqa: E731

    # exactness of the timed configuration against the plain kernel (itself pinned to the oracle)
    main_fn()
    torch.cuda.synchronize()
    if (d_status != 0).any() or not np.array_equal(d_out.cpu().numpy(), plain_out):
        raise SystemExit("scheduled batch differs from the plain kernel")

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    ms = timed_steps(main_fn, args.steps, args.warmup, stream, flush, nvtx="bench_timed")
    barrier()
    clk = clocks.stop()
    t_step = sum(ms) / len(ms)
    stats_main = ctx.last_stats()

    # comparison arms on the same batch
    k2 = max(3, args.steps // 2)
    ms_sorted = timed_steps(lambda: graphs["sorted"].launch(stream), k2, 1, stream, flush)
    stats_sorted = ctx.last_stats()
    ms_learned = timed_steps(lambda: graphs["learned"].launch(stream), k2, 1, stream, flush)
    stats_learned = ctx.last_stats()
    ms_plain = timed_steps(lambda: batch(g.SCHED_PLAIN), k2, 1, stream, flush)
    # The plain kernel over the jobs in length-sorted order (longest query first, then longest
    # target): the same one-block-per-job kernel, its blocks issued longest first so that the
    # batch's tail is made of short jobs.  The order is computed once on the host, outside the
    # timed region; the outputs come back in that order and are compared after un-permuting.
    perm = np.lexsort((-wl.jobs["tlen"].astype(np.int64), -wl.jobs["qlen"].astype(np.int64)))
    d_jobs_len = torch.from_numpy(np.ascontiguousarray(wl.jobs[perm]).view(np.uint8).copy()).to(dev)
    d_out_len = torch.zeros_like(d_out)

    def plain_sorted():
        ctx.extend_batch(sc, d_jobs_len, n, d_codes, d_nmask, d_out_len, d_status, mq, mt,
                         schedule=g.SCHED_PLAIN, stream=stream)

    plain_sorted()
    torch.cuda.synchronize()
    if (d_status != 0).any() or not np.array_equal(d_out_len.cpu().numpy(), plain_out[perm]):
        raise SystemExit("length-sorted plain batch differs from the plain kernel")
    ms_plain_len = timed_steps(plain_sorted, k2, 1, stream, flush)
    t_sorted, t_learned, t_plain, t_plain_len = (sum(x) / len(x) for x in (ms_sorted, ms_learned, ms_plain,
                                                                            ms_plain_len))

    # Per-class launch durations of the learned batch (the same kernels the graph replays),
    # each from CUDA events on the class's own stream, while the other classes run beside it.
    widths = np.array([t[0] for t in tiles], np.int64)
    member = np.searchsorted(widths, wl.jobs["qlen"].astype(np.int64), side="left")
    cls_jobs = np.bincount(member, minlength=len(tiles))
    cls_cells = np.bincount(member, weights=cells_np.astype(np.float64), minlength=len(tiles))
    # Algorithmic HBM bytes of each class's jobs: 24 B header + 2-bit query and target + their
    # N bits + 24 B of outputs per job.
    q64, t64 = wl.jobs["qlen"].astype(np.int64), wl.jobs["tlen"].astype(np.int64)
    job_bytes = 24 + (q64 + 3) // 4 + (t64 + 3) // 4 + (q64 + t64 + 7) // 8 + 24
    cls_bytes = np.bincount(member, weights=job_bytes.astype(np.float64), minlength=len(tiles))

    def class_table(schedule, mode):
        ctx.set_timing(mode)
        cls_ms = []
        for _ in range(3):
            flush.fill_(1)
            batch(schedule)
            cls_ms.append(ctx.class_times())
        ctx.set_timing(0)
        rows = []
        for k, t in enumerate(tiles):
            ms_k = [c[k][0] for c in cls_ms if c[k][0] >= 0]
            if cls_ms[-1][k][1] != int(cls_jobs[k]):
                raise SystemExit(f"class {k}: the library scheduled {cls_ms[-1][k][1]} jobs, qlen says {cls_jobs[k]}")
            if not ms_k:
                continue
            mk = sum(ms_k) / len(ms_k)
            rows.append({"width": int(t[0]), "kernel": kernel_name(t), "jobs": int(cls_jobs[k]),
                         "cells": int(cls_cells[k]), "ms": round(mk, 4),
                         "gcups": round(cls_cells[k] / (mk * 1e-3) / 1e9, 3),
                         "arith": "int16x2" if kernel_name(t) == "lane16" else "int32",
                         "alg_bytes": int(cls_bytes[k])})
        return rows

    # each class alone (its own kernel roofline), and side by side as the step runs them
    classes = class_table(g.SCHED_LEARNED, 2)
    classes_conc = class_table(g.SCHED_LEARNED, 1)
    ctx.set_tiles(tiles_of["sorted"])
    classes_sorted = class_table(g.SCHED_SORTED, 2)
    ctx.set_tiles(tiles)

    # end to end through the C ABI with host buffers (g3x_pipe): every step copies its job
    # stream and planes from pinned host memory, extends them with the same schedule and width
    # classes, and copies outputs and statuses back; a step's copies overlap its neighbours'
    # extension.  Timed over the K steps as a whole (the pipe keeps two batches in flight).
    bi = h_jobs.numel() + h_codes.numel() + h_nmask.numel()
    h_status = torch.zeros(n, dtype=torch.int32).pin_memory()
    bo = h_out.numel() * 4 + h_status.numel() * 4
    pipe = g.Pipe(ctx, sc, sched, n, h_codes.numel() // 4, h_nmask.numel() // 4)

    def e2e_step():
        pipe.submit(h_jobs, n, h_codes, h_nmask, mq, mt, h_out, h_status, stream)

    barrier()
    t_e2e = timed_pipeline(e2e_step, pipe.wait, args.steps, args.warmup, stream, flush)
    barrier()
    e2e_exact = bool((h_status == 0).all()) and np.array_equal(h_out.numpy(), plain_out)
    pipe.close()

    (t_step, t_e2e, t_plain, t_plain_len, t_sorted, t_learned), (tot_cells, tot_jobs) = combine_ranks(
        dist, [t_step, t_e2e, t_plain, t_plain_len, t_sorted, t_learned], [cells, n], dev)


    peak_ops = ctx.int_peak()
    if rank == 0:
        gcups = tot_cells / (t_step * 1e-3) / 1e9
        # cells/s rooflines: 8 int ops per cell; an int16x2 instruction does two cells
        peak32 = peak_ops / 8 / 1e9
        peak_of = {"int32": peak32, "int16x2": 2 * peak32}
        dom = max(classes, key=lambda c: c["ms"])
        dom_peak = peak_of[dom["arith"]]
        # the step against the blend of its classes' rooflines: the time every class's cells
        # would take at its own kernel's peak, over the measured step time
        ideal_ms = sum(c["cells"] / (peak_of[c["arith"]] * 1e9) * 1e3 for c in classes)
        tpj = TRAFFIC_PER_JOB.get(dom["width"]) if dom["kernel"] == "lane16" and args.workload == "cfg2" else None
        int16_cells = sum(c["cells"] for c in classes if c["arith"] == "int16x2")
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
                hbm_peak, hbm_src = float(json.load(fh)["hbm_gbs"]), "measured"
        except (OSError, ValueError, KeyError):
            hbm_peak, hbm_src = 6650.0, "fallback"
        kind, cpu_t, cpu_out = cpu_reference(wl, os.cpu_count() or 1)
        cpu_gcups = cells / cpu_t / 1e9
        idle = lambda s: round(s[1] / max(1, s[0] + s[1]), 4)  # noqa: E731
        gc = lambda t: round(tot_cells / (t * 1e-3) / 1e9, 3)  # noqa: E731
        line = {
            "metric": METRIC, "value": round(gcups, 3), "unit": "GCUPS", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int16x2 (int32 where the fit fails)" if int16_cells else "int32",
            "data": "synthetic (seeded generator, shapes of the benchmark configuration)",
            "config": bench_config(desc, n, cells),
            "setup": {"schedule": args.schedule if args.schedule != "auto" else "learned",
                      "launch": "one CUDA graph per step (features, MLP, counting sort, one persistent launch per width class)",
                      "width_classes": tiles, "width_classes_sorted": tiles_of["sorted"],
                      "max_qlen": mq, "max_tlen": mt, "int16x2_cell_frac": round(int16_cells / max(cells, 1), 4),
                      "l2": "256 MiB buffer written between timed steps", "parallelism": f"replicas x{ws}"},
            "extensions_per_s": round(tot_jobs / (t_step * 1e-3), 1),
            "arms": {"learned": {"gcups": gc(t_learned), "ms": round(t_learned, 4),
                                 "warp_idle_frac": idle(stats_learned)},
                     "sorted": {"gcups": gc(t_sorted), "ms": round(t_sorted, 4),
                                "warp_idle_frac": idle(stats_sorted),
                                "class_ms": [c["ms"] for c in classes_sorted]},
                     "plain_sorted": {"gcups": gc(t_plain_len), "ms": round(t_plain_len, 4),
                                      "kernel": "one 32-lane block per job, anti-diagonal wavefront, jobs by "
                                                "decreasing query then target length (host order, untimed)"},
                     "plain": {"gcups": gc(t_plain), "ms": round(t_plain, 4),
                               "kernel": "one 32-lane block per job, anti-diagonal wavefront, input order"}},
            "speedup_learned_vs_plain_sorted": round(t_plain_len / t_learned, 3),
            "speedup_learned_vs_plain": round(t_plain / t_learned, 3),
            "speedup_learned_vs_sorted": round(t_sorted / t_learned, 3),
            "cost_model": {**train_metrics, "prediction_on_this_batch": pred_err},
            "autotune_s": round(t_tune, 2),
            "e2e": {"value": gc(t_e2e), "unit": "GCUPS",
                    "ms_per_step": round(t_e2e, 4), "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                    "api": "g3x_pipe_submit per step (pinned host buffers; copies overlap the "
                           "neighbouring steps' extension), g3x_pipe_wait after the K steps",
                    "outputs_equal_plain_kernel": e2e_exact},
            "roofline": {"bound": "int_alu", "kernel": f"{dom['kernel']} (width class {dom['width']})",
                         "achieved": dom["gcups"], "peak": round(dom_peak, 3), "unit": "GCUPS",
                         "frac": round(dom["gcups"] / dom_peak, 4),
                         "traffic": None if tpj is None else int(tpj * dom["jobs"]),
                         "traffic_unit": "DRAM bytes per launch",
                         "traffic_source": "ncu dram__bytes_read + dram__bytes_write per job of this class "
                                           "(profiles/lane16_kernel_cfg2_class_traffic.md, 100k-seed case) x the "
                                           "class's jobs" if tpj is not None else None,
                         "alg_bytes": dom["alg_bytes"],
                         "algorithmic": "cells of the class launch (trip count of ksw.cu:346) / its "
                                        "CUDA-event duration, the class launched alone on the bench stream",
                         "peak_def": f"{dom['arith']} cells/s roofline: measured 32-bit int ops/s / 8 ops per "
                                     "cell" + (", x2 (two cells per int16x2 instruction)" if dom["arith"] == "int16x2" else ""),
                         "peak_source": "measured live: g3x_int_peak (DPX VIMNMX3 chains, 32-bit int ops/s)",
                         "int_ops_per_s": peak_ops, "int32_peak_gcups": round(peak32, 3),
                         "int16x2_peak_gcups": round(2 * peak32, 3),
                         "step_frac": round(ideal_ms / t_step, 4),
                         "step_frac_def": "sum over classes of cells / that class kernel's roofline, over the step time",
                         "class_ms_side_by_side": [c["ms"] for c in classes_conc],
                         "classes": classes},
            "hbm_job_stream": {"achieved_gbs": round(bi / (t_step * 1e-3) / 1e9, 2), "peak_gbs": hbm_peak,
                               "frac": round(bi / (t_step * 1e-3) / 1e9 / hbm_peak, 5),
                               "peak_source": hbm_src, "bytes_per_step": bi},
            "cpu_baseline": {"value": round(cpu_gcups, 4), "unit": "GCUPS", "cores": os.cpu_count(),
                             "kind": kind, "sample": f"whole rank-0 workload ({n} jobs), one pass",
                             "gpu_outputs_identical": bool(np.array_equal(cpu_out, plain_out))},
            "clocks": clk,
            # per step: the schedule (learned keys or length keys, scan, scatter) and one
            # persistent launch per width class
            "gpu_launches": args.steps * (3 + len(tiles)),
        }
        print(json.dumps(line), flush=True)
    for gr in graphs.values():
        gr.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
