"""Small profiling case: one synthetic batch extended a few times through one schedule.

    python -m g3sa_b200.profile_case --seed-stream [--units 2000000] [--chunk 262144]

runs the seed-level band-retry stream instead (config 5): the generator's seeds, the planes and
the regions in pinned host memory, g3x_extend_seeds_stream once with the plain kernel and once
through the width classes (tuned on a job batch of the same generator), both timed, their
regions compared.

    python -m g3sa_b200.profile_case [--kind 2] [--units 100000] [--schedule sorted|learned|plain]
                                     [--kernel auto] [--tiles WIDTH:LANES:TILE:WB:REFILL,...]
                                     [--reps 2] [--phase-clocks]

Generates the batch (the same seeded generator the benchmark uses), copies it to the GPU,
runs `reps` batches through g3x_ksw_extend2_batch and prints one line with the batch's
size and the last batch's time.  Nothing else runs on the GPU, so a profiler's launch
filters (-k, -s, -c) count only the extension's own kernels: per batch, the schedule's
sort kernels and one persistent launch per width class.

--phase-clocks runs the same batches through libg3x_phase.so (built by
`python -m g3sa_b200.build --phase-clocks`), whose int16x2 lane kernel adds up the clock cycles
its warps spend in each phase of the row loop, and prints, per width class of that kernel, the
cycles per warp row of each phase and their shares of the warp's time (the last batch only).
"""
import argparse
import ctypes
import os
import time

import numpy as np

import g3sa_b200 as g


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kind", type=int, default=2)
    ap.add_argument("--units", type=int, default=100000)
    ap.add_argument("--w", type=int, default=100)
    ap.add_argument("--unrelated", type=float, default=0.2)
    ap.add_argument("--schedule", default="sorted", choices=["plain", "sorted", "learned"])
    ap.add_argument("--kernel", default="auto", choices=["auto", "rolling", "rowpar", "lane"])
    ap.add_argument("--tiles", default="",
                    help="width classes of the sorted schedule, e.g. 20:4:5:1:1,288:1:0:0:8 "
                         "(lanes 1 = the lane-per-job kernel); default: the context's")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--class-times", action="store_true",
                    help="run the width classes one after another and print each one's time")
    ap.add_argument("--seed", type=int, default=0x6A5 + 2)
    ap.add_argument("--seed-stream", action="store_true")
    ap.add_argument("--chunk", type=int, default=262144)
    ap.add_argument("--phase-clocks", action="store_true")
    a = ap.parse_args()
    if a.phase_clocks:
        g.LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(g.__file__)), "libg3x_phase.so")
    if a.seed_stream:
        return seed_stream(a)
    import torch
    wl = g.synth(a.kind, a.units, seed=a.seed, w=a.w, unrelated=a.unrelated)
    codes, nmask = wl.planes()
    dev = torch.device("cuda", 0)
    d = [torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).copy()).to(dev)
         for x in (wl.jobs, codes, nmask)]
    out = torch.zeros((wl.n, 6), dtype=torch.int32, device=dev)
    status = torch.zeros(wl.n, dtype=torch.int32, device=dev)
    ctx = g.Context(0)
    if a.tiles:
        ctx.set_tiles([tuple(int(v) for v in c.split(":")) for c in a.tiles.split(",")])
    sched = {"plain": g.SCHED_PLAIN, "sorted": g.SCHED_SORTED, "learned": g.SCHED_LEARNED}[a.schedule]
    if sched == g.SCHED_LEARNED:     # the cost model on a held-out batch of the same generator
        from g3sa_b200 import learn
        learn.train(ctx, n_train=max(a.units // 2, 1000), seed_train=a.seed + 99, kind=a.kind, w=a.w,
                    unrelated=a.unrelated)
    kern = {"auto": g.KERNEL_AUTO, "rolling": g.KERNEL_ROLLING, "rowpar": g.KERNEL_ROWPAR,
            "lane": g.KERNEL_LANE}[a.kernel]
    mq, mt = int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max())
    if a.class_times:
        ctx.set_timing(2)
    dt = 0.0
    phase_read = None
    if a.phase_clocks:
        phase_read = g.lib().g3x_phase_clocks_read
        phase_read.argtypes = [ctypes.c_void_p, ctypes.c_int]
    clocks = np.zeros((8, 8), np.uint64)
    for _ in range(a.reps):
        if phase_read:
            phase_read(clocks.ctypes.data, 1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.extend_batch(g.default_score(), d[0], wl.n, d[1], d[2], out, status, mq, mt,
                         schedule=sched, kernel=kern)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    if a.class_times:
        print("class ms/jobs:", " ".join(f"{ms:.3f}/{jobs}" for ms, jobs in ctx.class_times()))
    bad = int((status != 0).sum())
    print(f"jobs {wl.n} max_qlen {mq} max_tlen {mt} last_batch_ms {dt * 1e3:.3f} job_errors {bad}")
    if phase_read:
        phase_read(clocks.ctypes.data, 0)
        names = ("refill", "row_begin", "blocks", "row_end", "output")
        for ci in range(8):
            rows = int(clocks[ci, 5])
            if rows == 0:
                continue
            tot = float(clocks[ci, :5].sum())
            print(f"qcap {32 * ci}-{32 * ci + 31}: warp rows {rows} blocks/row {clocks[ci, 6] / rows:.2f} "
                  f"cycles/row {tot / rows:.0f} | " +
                  " ".join(f"{nm} {clocks[ci, q] / rows:.0f} ({clocks[ci, q] / tot:.3f})" for q, nm in enumerate(names)))
    if bad:
        raise SystemExit(1)


def seed_stream(a):
    import torch
    units = a.units if a.units != 100000 else 2000000
    wl = g.synth(2, units, seed=a.seed, w=a.w, unrelated=a.unrelated)
    codes, nmask = wl.planes()
    ds = g.device_seeds(wl.seeds)
    n = len(ds)
    pin = lambda x: torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).copy()).pin_memory()  # noqa: E731
    h_seeds, h_codes, h_nmask = pin(ds), pin(codes), pin(nmask)
    h_regs = torch.zeros(n * g.REG_DT.itemsize, dtype=torch.uint8).pin_memory()
    h_status = torch.full((n,), 99, dtype=torch.int32).pin_memory()
    mq = int(wl.seeds["l_query"].max())
    mt = int((wl.seeds["rmax1"] - wl.seeds["rmax0"]).max())
    ctx = g.Context(0)
    tw = g.synth(2, 200000, seed=a.seed + 1, w=a.w, unrelated=a.unrelated)
    tc, tn = tw.planes()
    dev = torch.device("cuda", 0)
    td = [torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).copy()).to(dev) for x in (tw.jobs, tc, tn)]
    ctx.autotune(g.default_score(), td[0], tw.n, td[1], td[2], int(tw.jobs["qlen"].max()),
                 int(tw.jobs["tlen"].max()))
    opt = g.default_opt(w=a.w)
    regs = {}
    for name, sched, chunk in (("plain", g.SCHED_PLAIN, 65536), ("sorted", g.SCHED_SORTED, a.chunk)):
        dt = 0.0
        for _ in range(max(a.reps, 1)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.extend_seeds_stream(opt, h_seeds, h_codes, h_nmask, len(wl.u8), h_regs, h_status, mq, mt,
                                    chunk=chunk, schedule=sched)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
        if (h_status.numpy() != 0).any():
            raise SystemExit(f"{name}: seed errors")
        regs[name] = h_regs.numpy().view(g.REG_DT).copy()
        print(f"{name}: chunk {chunk} seeds {n} last_call_ms {dt * 1e3:.1f} seeds_per_s {n / dt:.4g}")
    same = all((regs["plain"][f] == regs["sorted"][f]).all()
               for f in ("rb", "re", "qb", "qe", "score", "truesc", "w"))
    print(f"regions identical: {same}")
    if not same:
        raise SystemExit(1)


if __name__ == "__main__":
    main()
