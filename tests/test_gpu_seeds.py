"""GPU seed-level extension with BWA's band retry (mem_chain2aln's extension block) against
the golden regions computed by the reference's own compiled mem_chain2aln lines, and the
chunked host-streaming form against the device form."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import golden_io, native as nat
from tests.gpu_util import run_seeds, ctx

pytestmark = pytest.mark.gpu
FIELDS = ["rb", "re", "qb", "qe", "score", "truesc", "w"]


def opt_from_cpu(cpu_opt):
    o = g.default_opt(w=int(cpu_opt["w"][0]), a=int(cpu_opt["a"][0]),
                      pen_clip5=int(cpu_opt["pen_clip5"][0]), pen_clip3=int(cpu_opt["pen_clip3"][0]))
    o["score"]["mat"] = cpu_opt["mat"]
    for f in ("o_del", "e_del", "o_ins", "e_ins", "zdrop"):
        o["score"][f] = cpu_opt[f]
    return o


@pytest.mark.parametrize("sched,lanes", [(g.SCHED_PLAIN, 0), (g.SCHED_SORTED, 8), (g.SCHED_SORTED, 16)])
@pytest.mark.parametrize("name", golden_io.seed_sets())
def test_seeds_match_golden(name, sched, lanes):
    u8, seeds, opt, reg = golden_io.load_seeds(name)
    regs, status = run_seeds(u8, seeds, opt_from_cpu(opt), sched, lanes)
    assert (status == 0).all()
    for f in FIELDS:
        bad = np.nonzero(regs[f] != reg[f])[0]
        assert bad.size == 0, f"{name} {f}: seeds {bad[:5]}"


def test_seeds_retry_counts_match_oracle():
    u8, seeds, opt, reg = golden_io.load_seeds("cfg5_w5")
    regs, status = run_seeds(u8, seeds, opt_from_cpu(opt))
    ref = nat.oracle_seeds(seeds, u8, opt)
    assert (regs["tries_left"] == ref["tries_left"]).all()
    assert (regs["tries_right"] == ref["tries_right"]).all()
    assert (regs["tries_left"] == 2).sum() + (regs["tries_right"] == 2).sum() > 10


@pytest.mark.parametrize("w", [100, 6])
def test_seeds_fresh_vs_oracle(w):
    wl = g.synth(2, 20000, seed=515 + w, w=w, unrelated=0.2)
    opt_cpu = nat.opt_from_score(g.default_score(), w=w)
    ref = nat.oracle_seeds(wl.seeds, wl.u8, opt_cpu)
    regs, status = run_seeds(wl.u8, wl.seeds, g.default_opt(w=w))
    assert (status == 0).all()
    for f in FIELDS:
        assert (regs[f] == ref[f]).all(), f


@pytest.mark.parametrize("chunk,pin", [(4096, True), (65536, True), (4096, False)])
def test_seeds_stream_matches_device_form(chunk, pin):
    """Pinned host buffers are copied straight to and from the device, pageable ones through the
    stream's pinned staging; both give the oracle's regions."""
    import torch
    wl = g.synth(2, 30000, seed=99, w=100, unrelated=0.2)
    codes, nmask = wl.planes()
    opt = g.default_opt(w=100)
    ds = g.device_seeds(wl.seeds)
    n = len(ds)
    host = (lambda t: t.pin_memory()) if pin else (lambda t: t)   # noqa: E731
    h_seeds = host(torch.from_numpy(ds.view(np.uint8).copy()))
    h_codes = host(torch.from_numpy(codes.view(np.uint8).copy()))
    h_nmask = host(torch.from_numpy(nmask.view(np.uint8).copy()))
    h_regs = host(torch.zeros(n * g.REG_DT.itemsize, dtype=torch.uint8))
    h_status = host(torch.full((n,), 99, dtype=torch.int32))
    mq = int(wl.seeds["l_query"].max())
    mt = int((wl.seeds["rmax1"] - wl.seeds["rmax0"]).max())

    class _H:  # host array with the length of the seed list
        def __init__(self, t, n):
            self.t, self.n = t, n

        def __len__(self):
            return self.n

        def data_ptr(self):
            return self.t.data_ptr()

    ctx().extend_seeds_stream(opt, _H(h_seeds, n), h_codes, h_nmask, len(wl.u8), h_regs, h_status,
                              mq, mt, chunk=chunk)
    regs = h_regs.numpy().view(g.REG_DT)
    status = h_status.numpy()
    ref = nat.oracle_seeds(wl.seeds, wl.u8, nat.opt_from_score(g.default_score(), w=100))
    assert (status == 0).all()
    for f in FIELDS:
        assert (regs[f] == ref[f]).all(), f


@pytest.mark.parametrize("sched", [g.SCHED_SORTED, g.SCHED_LEARNED])
def test_seeds_through_lane_classes(sched):
    """Each wave of the seed-level call sorted into width classes that run the lane-per-job
    kernels (int32, int16x2, ring), length-sorted or by a model's predictions."""
    import torch
    from tests.gpu_util import to_dev
    wl = g.synth(2, 20000, seed=0x5EED5, w=100, unrelated=0.2)
    opt_cpu = nat.opt_from_score(g.default_score(), w=100)
    ref = nat.oracle_seeds(wl.seeds, wl.u8, opt_cpu)
    c = g.Context(0)
    c.set_tiles([(16, 1, 2, 0, 32), (56, 1, 0, 0, 32), (128, 1, 2, 0, 8), (176, 1, 432, 0, 1),
                 (1 << 30, 32, 9, 0, 1)])
    if sched == g.SCHED_LEARNED:
        c.mlp_init(3)
        c.mlp_set_params(c.mlp_params())
    codes, nmask = wl.planes()
    ds = g.device_seeds(wl.seeds)
    n = len(ds)
    d_seeds, d_codes, d_nmask = to_dev(ds), to_dev(codes), to_dev(nmask)
    d_regs = torch.zeros(n * g.REG_DT.itemsize, dtype=torch.uint8, device="cuda")
    d_status = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    mq = int(wl.seeds["l_query"].max())
    mt = int((wl.seeds["rmax1"] - wl.seeds["rmax0"]).max())
    c.extend_seeds(g.default_opt(w=100), d_seeds, n, d_codes, d_nmask, d_regs, d_status, mq, mt, sched, 0)
    torch.cuda.synchronize()
    regs = d_regs.cpu().numpy().view(g.REG_DT)
    assert (d_status.cpu().numpy() == 0).all()
    for f in FIELDS:
        assert (regs[f] == ref[f]).all(), f
