"""Small profiling case: one synthetic batch extended a few times through one schedule.

    python -m g3sa_b200.profile_case [--kind 2] [--units 100000] [--schedule sorted]
                                     [--kernel auto] [--tiles WIDTH:LANES:TILE:WB:REFILL,...]
                                     [--reps 2]

Generates the batch (the same seeded generator the benchmark uses), copies it to the GPU,
runs `reps` batches through g3x_ksw_extend2_batch and prints one line with the batch's
size and the last batch's time.  Nothing else runs on the GPU, so a profiler's launch
filters (-k, -s, -c) count only the extension's own kernels: per batch, the schedule's
sort kernels and one persistent launch per width class.
"""
import argparse
import time

import numpy as np

import g3sa_b200 as g


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kind", type=int, default=2)
    ap.add_argument("--units", type=int, default=100000)
    ap.add_argument("--w", type=int, default=100)
    ap.add_argument("--unrelated", type=float, default=0.2)
    ap.add_argument("--schedule", default="sorted", choices=["plain", "sorted"])
    ap.add_argument("--kernel", default="auto", choices=["auto", "rolling", "rowpar", "lane"])
    ap.add_argument("--tiles", default="",
                    help="width classes of the sorted schedule, e.g. 20:4:5:1:1,288:1:0:0:8 "
                         "(lanes 1 = the lane-per-job kernel); default: the context's")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--class-times", action="store_true",
                    help="run the width classes one after another and print each one's time")
    ap.add_argument("--seed", type=int, default=0x6A5 + 2)
    a = ap.parse_args()
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
    sched = {"plain": g.SCHED_PLAIN, "sorted": g.SCHED_SORTED}[a.schedule]
    kern = {"auto": g.KERNEL_AUTO, "rolling": g.KERNEL_ROLLING, "rowpar": g.KERNEL_ROWPAR,
            "lane": g.KERNEL_LANE}[a.kernel]
    mq, mt = int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max())
    if a.class_times:
        ctx.set_timing(2)
    dt = 0.0
    for _ in range(a.reps):
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
    if bad:
        raise SystemExit(1)


if __name__ == "__main__":
    main()
