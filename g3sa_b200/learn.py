"""Training workflow of the learned cost model (host orchestration over the C ABI).

Traces come from the method itself: a held-out synthetic batch of the workload to be scheduled
(same generator kind, another seed) is extended by the plain kernel, whose per-job cell counters are the targets
(log2(1 + cells)); the features come from the library's feature kernel; the 5 -> 64 -> 64 -> 1
MLP is trained on the GPU by the library's own forward/backward/Adam kernels
(g3x_mlp_train).  Everything runs on the device; only the loss curve comes back.
"""
import time

import numpy as np

import g3sa_b200 as g


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def traces(ctx, n, seed, kind=1, w=100, unrelated=0.2, score=None):
    """(features [m,5] device, targets [m] device, cells numpy) from the m jobs the generator
    `kind` makes for n units (jobs for kind 1, seeds for kind 2, segments for kind 4)."""
    import torch
    score = g.default_score() if score is None else score
    wl = g.synth(kind, n, seed=seed, w=w, unrelated=unrelated)
    codes, nmask = wl.planes()
    d_jobs, d_codes, d_nmask = _dev(wl.jobs), _dev(codes), _dev(nmask)
    out = torch.zeros((wl.n, 6), dtype=torch.int32, device="cuda")
    status = torch.zeros(wl.n, dtype=torch.int32, device="cuda")
    cells = torch.zeros(wl.n, dtype=torch.int32, device="cuda")
    ctx.extend_batch(score, d_jobs, wl.n, d_codes, d_nmask, out, status,
                     int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max()),
                     schedule=g.SCHED_PLAIN, d_cells=cells)
    feat = torch.zeros((wl.n, g.MLP_FEATURES), dtype=torch.float32, device="cuda")
    ctx.features(d_jobs, wl.n, d_codes, d_nmask, feat)
    target = torch.log2(1.0 + cells.to(torch.float32))
    torch.cuda.synchronize()
    if (status != 0).any():
        raise RuntimeError("trace run reported job errors")
    return feat, target, cells.cpu().numpy()


def lr_schedule(lr, epochs):
    """The learning rate of each epoch: lr for the first two, then halved every epoch."""
    return [lr * 0.5 ** max(0, e - 1) for e in range(epochs)]


def train(ctx, n_train=2_000_000, seed_train=0xA11CE, epochs=5, batch=4096, lr=2e-3, init_seed=17,
          kind=1, w=100, unrelated=0.2):
    """Trains the context's model on the traces of n_train generator units, one g3x_mlp_train
    call per epoch (the Adam state carries over) with the rate of lr_schedule; returns a
    metrics dict."""
    t0 = time.perf_counter()
    feat, target, _ = traces(ctx, n_train, seed_train, kind=kind, w=w, unrelated=unrelated)
    m = int(target.shape[0])
    t1 = time.perf_counter()
    ctx.mlp_init(init_seed)
    rates = lr_schedule(lr, epochs)
    losses = [float(ctx.mlp_train(feat, target, m, 1, batch, r, seed=init_seed + e)[0])
              for e, r in enumerate(rates)]
    t2 = time.perf_counter()
    return {"traces": m, "trace_kind": kind, "trace_s": round(t1 - t0, 3), "train_s": round(t2 - t1, 3),
            "epochs": epochs, "batch": batch, "lr": [round(r, 6) for r in rates],
            "loss_curve": [round(x, 5) for x in losses], "params": g.MLP_PARAMS}


def prediction_error(ctx, d_jobs, n, d_codes, d_nmask, cells):
    """Per-job cell-count prediction error of the trained model on a batch whose measured
    cells are `cells` (numpy): median / mean absolute relative error and log2 MAE."""
    import torch
    feat = torch.zeros((n, g.MLP_FEATURES), dtype=torch.float32, device="cuda")
    pred = torch.zeros(n, dtype=torch.float32, device="cuda")
    ctx.features(d_jobs, n, d_codes, d_nmask, feat)
    ctx.mlp_predict(feat, n, pred)
    torch.cuda.synchronize()
    p = pred.cpu().numpy().astype(np.float64)
    c = cells.astype(np.float64)
    est = np.exp2(p) - 1.0
    rel = np.abs(est - c) / np.maximum(c, 1.0)
    return {"median_rel_err": round(float(np.median(rel)), 4),
            "mean_rel_err": round(float(np.mean(np.minimum(rel, 10.0))), 4),
            "log2_mae": round(float(np.mean(np.abs(p - np.log2(1.0 + c)))), 4),
            "corr_log2": round(float(np.corrcoef(p, np.log2(1.0 + c))[0, 1]), 4)}
