"""The pipelined host-batch API (g3x_pipe): batches in host memory, copies overlapped with the
neighbouring batches' extension.  Results must equal the oracle's bit for bit whatever the
order of submits, set reuse and batch sizes; sizes beyond the pipe's are rejected."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import native as nat
from tests.gpu_util import ctx

pytestmark = pytest.mark.gpu


def _batches():
    out = []
    for k, (kind, n, w) in enumerate([(2, 6000, 100), (1, 9000, 100), (2, 3000, 50), (1, 2000, 100)]):
        wl = g.synth(kind, n, seed=0x91E + 17 * k, w=w, unrelated=0.2 if kind == 2 else 0.0)
        codes, nmask = wl.planes()
        out.append((wl, np.ascontiguousarray(codes), np.ascontiguousarray(nmask)))
    return out


@pytest.mark.parametrize("schedule", [g.SCHED_SORTED, g.SCHED_PLAIN])
def test_pipe_matches_oracle(schedule):
    import torch
    sc = g.default_score()
    batches = _batches()
    mj = max(b[0].n for b in batches)
    mc = max(len(b[1]) for b in batches)
    mn = max(len(b[2]) for b in batches)
    pipe = g.Pipe(ctx(), sc, schedule, mj, mc, mn)
    stream = torch.cuda.Stream()
    res = []
    for wl, codes, nmask in batches:   # four submits: both sets are reused once
        h_jobs = torch.from_numpy(wl.jobs.view(np.uint8).copy()).pin_memory()
        h_codes = torch.from_numpy(codes.view(np.uint8).copy()).pin_memory()
        h_nmask = torch.from_numpy(nmask.view(np.uint8).copy()).pin_memory()
        h_out = torch.full((wl.n, 6), -777, dtype=torch.int32).pin_memory()
        h_status = torch.full((wl.n,), 99, dtype=torch.int32).pin_memory()
        pipe.submit(h_jobs, wl.n, h_codes, h_nmask, int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max()),
                    h_out, h_status, stream)
        res.append((h_jobs, h_codes, h_nmask, h_out, h_status))
    pipe.wait(stream)
    stream.synchronize()
    for (wl, _, _), (_, _, _, h_out, h_status) in zip(batches, res):
        ref, _, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
        assert (h_status.numpy() == 0).all()
        bad = np.nonzero((h_out.numpy() != ref).any(1))[0]
        assert bad.size == 0, f"jobs {bad[:5]}"
    pipe.close()


def test_pipe_rejects_oversize_and_accepts_empty():
    import torch
    sc = g.default_score()
    wl = g.synth(1, 500, seed=7)
    codes, nmask = wl.planes()
    pipe = g.Pipe(ctx(), sc, g.SCHED_SORTED, wl.n - 1, len(codes), len(nmask))
    out = np.zeros((wl.n, 6), np.int32)
    status = np.zeros(wl.n, np.int32)
    with pytest.raises(g.G3xError):
        pipe.submit(wl.jobs, wl.n, codes, nmask, 200, 400, out, status)
    pipe.submit(wl.jobs, 0, codes, nmask, 200, 400, out, status)   # nothing to do
    pipe.wait()
    torch.cuda.synchronize()
    pipe.close()
    with pytest.raises(g.G3xError):
        g.Pipe(ctx(), sc, 7, 10, 10, 10)
