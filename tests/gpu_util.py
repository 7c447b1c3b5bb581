"""Helpers for the GPU tests: run batches through the C ABI with torch-owned device buffers."""
import numpy as np

import g3sa_b200 as g

_ctx = None


def ctx():
    global _ctx
    if _ctx is None:
        _ctx = g.Context(0)
    return _ctx


def to_dev(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.uint8).copy()).cuda()


def run_batch(u8, jobs, score, schedule=g.SCHED_PLAIN, lanes=0, max_qlen=None, max_tlen=None,
              tile=0, kernel=g.KERNEL_AUTO, n_bases=None, with_rows=False):
    """Returns (ext[n,6], status[n], cells[n]) from the GPU, and rows[n] after them with
    with_rows."""
    import torch
    n = len(jobs)
    codes, nmask = g.pack_planes(u8)
    d_jobs, d_codes, d_nmask = to_dev(jobs), to_dev(codes), to_dev(nmask)
    out = torch.full((n, 6), -777, dtype=torch.int32, device="cuda")
    status = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    cells = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    rows = torch.full((n,), -1, dtype=torch.int32, device="cuda") if with_rows else None
    mq = int(jobs["qlen"].max()) if max_qlen is None else max_qlen
    mt = int(jobs["tlen"].max()) if max_tlen is None else max_tlen
    ctx().extend_batch(score, d_jobs, n, d_codes, d_nmask, out, status, mq, mt,
                       schedule=schedule, lanes=lanes, d_cells=cells, tile=tile, kernel=kernel,
                       n_bases=n_bases, d_rows=rows)
    torch.cuda.synchronize()
    res = (out.cpu().numpy(), status.cpu().numpy(), cells.cpu().numpy())
    return res + (rows.cpu().numpy(),) if with_rows else res


def run_seeds(u8, seeds, opt, schedule=g.SCHED_SORTED, lanes=0, n_bases=None):
    """Seed-level extension on the GPU: returns (regs REG_DT, status)."""
    import torch
    codes, nmask = g.pack_planes(u8)
    ds = g.device_seeds(seeds)
    n = len(ds)
    d_seeds, d_codes, d_nmask = to_dev(ds), to_dev(codes), to_dev(nmask)
    d_regs = torch.zeros(n * g.REG_DT.itemsize, dtype=torch.uint8, device="cuda")
    d_status = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    mq = int(seeds["l_query"].max())
    mt = int((seeds["rmax1"] - seeds["rmax0"]).max())
    ctx().extend_seeds(opt, d_seeds, n, d_codes, d_nmask, d_regs, d_status, mq, mt, schedule, lanes,
                       n_bases=n_bases)
    torch.cuda.synchronize()
    return d_regs.cpu().numpy().view(g.REG_DT), d_status.cpu().numpy()
