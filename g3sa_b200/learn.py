"""Training workflow of the learned cost model (host orchestration over the C ABI).

Traces come from the method itself: a held-out synthetic batch of the workload to be scheduled
(same generator kind, another seed) is extended by the plain kernel, whose per-job row counters
give the targets; the features come from the library's feature kernel; the 5 -> 64 -> 64 -> 1
MLP is trained on the GPU by the library's own forward/backward/Adam kernels (g3x_mlp_train).

The target is a correction to the length-sorted schedule's row bound: log2(1 + rows) less
log2(1 + tlen), rows the trips of the row loop of ksw.cu:346 (the z-drop or an empty band ends
it early).  A job that runs to its last row has a correction of exactly 0, whatever its length,
so the network only learns where the z-drop ends a job early (a behaviour that looks the same at
every length), and the scheduler, which adds min(0, prediction + 1) back onto log2(1 + tlen),
keeps the length order wherever the network sees no end before half the rows.  Rows, not cells,
because a row-synchronous warp runs as many steps as its longest job has rows.
"""
import time

import numpy as np

import g3sa_b200 as g


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def row_target(rows, tlen):
    """The model's target: log2(1 + rows) - log2(1 + tlen) (numpy or torch, float32), <= 0."""
    if hasattr(rows, "to"):
        import torch
        return torch.log2(1.0 + rows.to(torch.float32)) - torch.log2(1.0 + tlen.to(torch.float32))
    return (np.log2(1.0 + rows.astype(np.float64)) - np.log2(1.0 + tlen.astype(np.float64))).astype(np.float32)


def traces(ctx, n, seed, kind=1, w=100, unrelated=0.2, score=None, with_jobs=False):
    """(features [m,5] device, targets [m] device, cells numpy) from the m jobs the generator
    `kind` makes for n units (jobs for kind 1, seeds for kind 2, segments for kind 4); the
    targets are row_target of the plain kernel's row counts."""
    import torch
    score = g.default_score() if score is None else score
    wl = g.synth(kind, n, seed=seed, w=w, unrelated=unrelated)
    codes, nmask = wl.planes()
    d_jobs, d_codes, d_nmask = _dev(wl.jobs), _dev(codes), _dev(nmask)
    out = torch.zeros((wl.n, 6), dtype=torch.int32, device="cuda")
    status = torch.zeros(wl.n, dtype=torch.int32, device="cuda")
    cells = torch.zeros(wl.n, dtype=torch.int32, device="cuda")
    rows = torch.zeros(wl.n, dtype=torch.int32, device="cuda")
    ctx.extend_batch(score, d_jobs, wl.n, d_codes, d_nmask, out, status,
                     int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max()),
                     schedule=g.SCHED_PLAIN, d_cells=cells, d_rows=rows)
    feat = torch.zeros((wl.n, g.MLP_FEATURES), dtype=torch.float32, device="cuda")
    ctx.features(d_jobs, wl.n, d_codes, d_nmask, feat)
    tlen = torch.from_numpy(wl.jobs["tlen"].astype(np.int32)).cuda()
    target = row_target(rows, tlen)
    torch.cuda.synchronize()
    if (status != 0).any():
        raise RuntimeError("trace run reported job errors")
    if with_jobs:
        return feat, target, cells.cpu().numpy(), wl.jobs, (d_jobs, d_codes, d_nmask)
    return feat, target, cells.cpu().numpy()


def lr_schedule(lr, epochs):
    """The learning rate of each epoch: lr for the first two, then halved every epoch."""
    return [lr * 0.5 ** max(0, e - 1) for e in range(epochs)]


# The learned schedule is kept only if, on the training traces, its order saves at least this
# fraction of the warps' row work against the length order (warp_work); otherwise the length order
# is already as good and the context falls back to it without running the inference.
MIN_GAIN = 0.03


def sort_keys(jobs, score, tiles, corr=None):
    """The counting sort's key of each job (g3x_sched.cu cost_kernel): width class, then row bin
    (log2(1 + tlen), plus min(0, corr + 1) when learned), then row-width bin."""
    q = jobs["qlen"].astype(np.int64)
    t = jobs["tlen"].astype(np.int64)
    mat = np.asarray(score["mat"]).reshape(-1)
    max_sc, eb = int(mat.max()), int(score["end_bonus"][0])
    w = jobs["w"].astype(np.int64)
    for o, e in ((int(score["o_ins"][0]), int(score["e_ins"][0])), (int(score["o_del"][0]), int(score["e_del"][0]))):
        num = q * max_sc + eb - o
        w = np.minimum(w, np.maximum(np.where(num >= 0, num // e + 1, 1), 1))
    wide = np.minimum(q, 2 * w + 1)
    widths = np.array([tw[0] for tw in tiles], np.int64)
    cls = np.minimum(np.searchsorted(widths, q, side="left"), len(widths) - 1)
    lr = np.log2(1.0 + t)
    if corr is not None:
        lr = lr + np.minimum(corr + 1.0, 0.0)
    rb = np.clip(((16.0 - lr) * 4.0).astype(np.int64), 0, 63)
    wb = 31 - np.minimum((wide + 7) >> 3, 31)
    return cls * 2048 + rb * 32 + wb, cls, np.maximum((wide + 7) >> 3, 1)


def warp_work(keys, cls, rows, blocks):
    """Row work of warps that take 32 consecutive jobs of a width class in key order: per warp,
    its longest job's rows times its widest job's row blocks (a row-synchronous warp's cost)."""
    o = np.argsort(keys, kind="stable")
    c, r, b = cls[o], rows[o].astype(np.int64), blocks[o].astype(np.int64)
    total = 0
    for k in np.unique(c):
        sel = c == k
        rk, bk = r[sel], b[sel]
        pad = (-len(rk)) % 32
        rk = np.concatenate([rk, np.zeros(pad, np.int64)]).reshape(-1, 32)
        bk = np.concatenate([bk, np.zeros(pad, np.int64)]).reshape(-1, 32)
        total += int((rk.max(1) * bk.max(1)).sum())
    return total


def train(ctx, n_train=2_000_000, seed_train=0xA11CE, epochs=5, batch=4096, lr=2e-3, init_seed=17,
          kind=1, w=100, unrelated=0.2):
    """Trains the context's model on the traces of n_train generator units, one g3x_mlp_train
    call per epoch (the Adam state carries over) with the rate of lr_schedule, and makes the
    learned schedule consult it only if its order saves at least MIN_GAIN of the warps' row work
    on those traces against the length order, with the context's width classes
    (g3x_mlp_set_active); returns a metrics dict."""
    t0 = time.perf_counter()
    feat, target, _, jobs, (d_jobs, d_codes, d_nmask) = traces(ctx, n_train, seed_train, kind=kind, w=w,
                                                               unrelated=unrelated, with_jobs=True)
    m = int(target.shape[0])
    t1 = time.perf_counter()
    ctx.mlp_init(init_seed)
    rates = lr_schedule(lr, epochs)
    losses = [float(ctx.mlp_train(feat, target, m, 1, batch, r, seed=init_seed + e)[0])
              for e, r in enumerate(rates)]
    t2 = time.perf_counter()
    import torch
    # the corrections the learned schedule itself would apply (its bf16 network and the
    # near-diagonal check), so that the simulated order is the one it would run
    pred = torch.zeros(m, dtype=torch.float32, device="cuda")
    ctx.mlp_predict_jobs(d_jobs, m, d_codes, d_nmask, pred)
    corr = pred.cpu().numpy().astype(np.float64)
    tl = jobs["tlen"].astype(np.float64)
    rows = np.rint(np.exp2(target.cpu().numpy().astype(np.float64) + np.log2(1.0 + tl)) - 1.0)
    score, tiles = g.default_score(), ctx.get_tiles()
    k_sorted, cls, blocks = sort_keys(jobs, score, tiles)
    k_learned, _, _ = sort_keys(jobs, score, tiles, corr)
    work_sorted, work_learned = warp_work(k_sorted, cls, rows, blocks), warp_work(k_learned, cls, rows, blocks)
    gain = 1.0 - work_learned / max(work_sorted, 1)
    ctx.mlp_set_active(gain >= MIN_GAIN)
    return {"traces": m, "trace_kind": kind, "trace_s": round(t1 - t0, 3), "train_s": round(t2 - t1, 3),
            "epochs": epochs, "batch": batch, "lr": [round(r, 6) for r in rates],
            "loss_curve": [round(x, 5) for x in losses], "params": g.MLP_PARAMS,
            "warp_work_gain_on_traces": round(gain, 4), "active": bool(gain >= MIN_GAIN)}


def prediction_error(ctx, jobs, d_jobs, n, d_codes, d_nmask, rows):
    """Per-job row-count prediction error of the trained model on a batch (host jobs `jobs`,
    device copy d_jobs) whose measured row counts are `rows` (numpy): log2(1 + tlen) plus the
    model's correction is its log2(1 + rows) estimate; median / mean absolute relative error
    (the mean with each job's error capped at 10), log2 MAE and the log2 correlation."""
    import torch
    feat = torch.zeros((n, g.MLP_FEATURES), dtype=torch.float32, device="cuda")
    pred = torch.zeros(n, dtype=torch.float32, device="cuda")
    ctx.features(d_jobs, n, d_codes, d_nmask, feat)
    ctx.mlp_predict(feat, n, pred)
    torch.cuda.synchronize()
    c = pred.cpu().numpy().astype(np.float64)
    p = c + np.log2(1.0 + jobs["tlen"].astype(np.float64))
    r = rows.astype(np.float64)
    est = np.exp2(p) - 1.0
    rel = np.abs(est - r) / np.maximum(r, 1.0)
    return {"quantity": "rows of the row loop (ksw.cu:346) per job",
            "median_rel_err": round(float(np.median(rel)), 4),
            "mean_rel_err": round(float(np.mean(np.minimum(rel, 10.0))), 4),
            "log2_mae": round(float(np.mean(np.abs(p - np.log2(1.0 + r)))), 4),
            "corr_log2": round(float(np.corrcoef(p, np.log2(1.0 + r))[0, 1]), 4)}
