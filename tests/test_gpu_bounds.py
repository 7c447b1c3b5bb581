"""Job headers against the planes, and the plain kernel's bounded step count, on the GPU.

A job whose query or target reaches past the bases the planes hold (the batch options'
n_bases) gets the per-job status G3X_ERR_INVALID and zero outputs from every kernel -- the
kernels refuse it before any of its bases is read -- while the other jobs of the batch keep the
oracle's outputs; a seed whose read or window reaches past the planes gets G3X_ERR_INVALID from
the seed driver.  The plain kernel's per-job step bound (which a correct run never reaches) can be
lowered with g3x_set_step_limit: jobs that run out end with G3X_ERR_TIMEOUT, the batch completes,
and the context's next batch is exact again."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import native as nat
from tests.gpu_util import ctx, run_batch, run_seeds

pytestmark = pytest.mark.gpu

LANE_TILES = {  # width classes of one lane kernel each, the row-parallel kernel last
    "lane": [(64, 1, 0, 0, 8), (232, 1, 0, 0, 8), (1 << 30, 32, 9, 0, 1)],
    "lane16": [(64, 1, 2, 0, 8), (232, 1, 2, 0, 8), (1 << 30, 32, 9, 0, 1)],
    "lane2": [(64, 1, 4, 0, 8), (232, 1, 4, 0, 8), (1 << 30, 32, 9, 0, 1)],
}


def broken_jobs(seed):
    """Seeded jobs on planes of exactly len(u8) bases, with some queries and targets moved to
    end past those bases (by one base, by many, and past 2^32)."""
    wl = g.synth(2, 2000, seed=seed, w=100, unrelated=0.2)
    n_bases = len(wl.u8)
    jobs = wl.jobs.copy()
    k = np.arange(len(jobs))
    bq = (k % 7 == 3) & (jobs["qlen"] > 0)
    bt = (k % 11 == 5) & (jobs["tlen"] > 0) & ~bq
    q, t = jobs["qlen"].astype(np.int64), jobs["tlen"].astype(np.int64)
    jobs["q_off"][bq] = n_bases - q[bq] + 1
    jobs["t_off"][bt] = n_bases - t[bt] + 1 + (k[bt] % 3) * 1000
    far = k % 97 == 50
    jobs["q_off"][far] = 0xFFFFFFF0
    bad = bq | bt | far
    return wl, jobs, n_bases, bad


def check(out, status, cells, ref, rcells, bad):
    assert (status[bad] == g.G3X_ERR_INVALID).all()
    assert (out[bad] == 0).all() and (cells[bad] == 0).all()
    assert (status[~bad] == 0).all()
    np.testing.assert_array_equal(out[~bad], ref[~bad])
    np.testing.assert_array_equal(cells[~bad], rcells[~bad])


@pytest.mark.parametrize("schedule", [g.SCHED_PLAIN, g.SCHED_SORTED, g.SCHED_LEARNED])
def test_jobs_past_the_planes_are_refused(schedule):
    wl, jobs, n_bases, bad = broken_jobs(0xB0D)
    sc = g.default_score()
    if schedule == g.SCHED_LEARNED:       # the learned path reads the planes for its features too
        c = ctx()
        c.mlp_init(3)
        c.mlp_set_params(c.mlp_params())
    ref, rcells, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
    out, status, cells = run_batch(wl.u8, jobs, sc, schedule, n_bases=n_bases,
                                   max_qlen=int(jobs["qlen"].max()), max_tlen=int(jobs["tlen"].max()))
    check(out, status, cells, ref, rcells, bad)


@pytest.mark.parametrize("kind", sorted(LANE_TILES))
def test_lane_kernels_refuse_jobs_past_the_planes(kind):
    wl, jobs, n_bases, bad = broken_jobs(0xB0E)
    sc = g.default_score()
    c = ctx()
    tiles = c.get_tiles()
    try:
        c.set_tiles(LANE_TILES[kind])
        ref, rcells, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
        out, status, cells = run_batch(wl.u8, jobs, sc, g.SCHED_SORTED, n_bases=n_bases)
        check(out, status, cells, ref, rcells, bad)
    finally:
        c.set_tiles(tiles)


def test_seeds_past_the_planes_are_refused():
    wl = g.synth(2, 1500, seed=0xB0F, w=100, unrelated=0.2)
    n_bases = len(wl.u8)
    seeds = wl.seeds.copy()
    k = np.arange(len(seeds))
    br = k % 9 == 4
    bw = (k % 13 == 6) & ~br
    seeds["read_off"][br] = n_bases - seeds["l_query"][br].astype(np.int64) + 2
    seeds["win_off"][bw] = n_bases - (seeds["rmax1"][bw] - seeds["rmax0"][bw]).astype(np.int64) + 1
    ref = nat.oracle_seeds(wl.seeds, wl.u8, nat.opt_from_score(g.default_score(), w=100))
    regs, status = run_seeds(wl.u8, seeds, g.default_opt(w=100), n_bases=n_bases)
    bad = br | bw
    assert (status[bad] == g.G3X_ERR_INVALID).all()
    assert (status[~bad] == 0).all()
    for f in ("rb", "re", "qb", "qe", "score", "truesc", "w"):
        np.testing.assert_array_equal(regs[f][~bad], ref[f][~bad])


def test_plain_kernel_step_limit_ends_jobs_with_timeout():
    wl = g.synth(1, 3000, seed=0x71, w=100, unrelated=0.2)
    sc = g.default_score()
    ref, rcells, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
    c = ctx()
    try:
        c.set_step_limit(40)
        out, status, _ = run_batch(wl.u8, wl.jobs, sc, g.SCHED_PLAIN)
        assert set(np.unique(status)) <= {0, g.G3X_ERR_TIMEOUT}
        assert (status == g.G3X_ERR_TIMEOUT).sum() > 100         # jobs that need more steps
        ok = status == 0
        np.testing.assert_array_equal(out[ok], ref[ok])          # the short ones finish exactly
    finally:
        c.set_step_limit(0)
    out, status, cells = run_batch(wl.u8, wl.jobs, sc, g.SCHED_PLAIN)
    assert (status == 0).all()
    np.testing.assert_array_equal(out, ref)
    np.testing.assert_array_equal(cells, rcells)


def move_past(jobs, n_bases):
    """Some queries and targets moved to end one base or more past n_bases bases; their mask."""
    jobs = jobs.copy()
    k = np.arange(len(jobs))
    q, t = jobs["qlen"].astype(np.int64), jobs["tlen"].astype(np.int64)
    bq = (k % 5 == 1) & (q > 0)
    bt = (k % 7 == 2) & (t > 0) & ~bq
    jobs["q_off"][bq] = n_bases - q[bq] + 1
    jobs["t_off"][bt] = n_bases - t[bt] + 1 + (k[bt] % 4) * 500
    return jobs, bq | bt


def test_global_alignment_refuses_jobs_past_the_planes():
    import torch
    from tests.gpu_util import to_dev
    cj, u8 = nat.global_jobs(2000, 31, max_len=160)
    stride = int((cj["qlen"] + cj["tlen"]).max()) + 2
    s_o, c_o, n_o, _ = nat.oracle_global(cj, u8, g.default_score(), stride)
    jobs = np.zeros(len(cj), g.JOB_DT)
    for f in ("q_off", "t_off", "qlen", "tlen", "w"):
        jobs[f] = cj[f]
    jobs, bad = move_past(jobs, len(u8))
    n = len(jobs)
    codes, nmask = g.pack_planes(u8)
    d_score = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_cig = torch.zeros(n * stride, dtype=torch.int32, device="cuda")
    d_nc = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_st = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    ctx().global_batch(g.default_score(), to_dev(jobs), n, to_dev(codes), to_dev(nmask), int(jobs["qlen"].max()),
                       int(jobs["tlen"].max()), int(jobs["w"].max()), d_score, d_cig, stride, d_nc, d_st,
                       n_bases=len(u8))
    torch.cuda.synchronize()
    st, sc_, nc = d_st.cpu().numpy(), d_score.cpu().numpy(), d_nc.cpu().numpy()
    assert (st[bad] == g.G3X_ERR_INVALID).all() and (nc[bad] == 0).all()
    assert (st[~bad] == 0).all()
    np.testing.assert_array_equal(sc_[~bad], s_o[~bad])
    np.testing.assert_array_equal(nc[~bad], n_o[~bad])


def test_striped_alignment_refuses_jobs_past_the_planes():
    import torch
    from tests.gpu_util import to_dev
    cj, u8 = nat.sw_jobs(2000, 41)
    sc = g.default_score()
    want, _ = nat.oracle_sw(cj, u8, sc, g.KSW_XSTART)
    jobs = np.zeros(len(cj), g.JOB_DT)
    for f in ("q_off", "t_off", "qlen", "tlen", "flags"):
        jobs[f] = cj[f]
    jobs, bad = move_past(jobs, len(u8))
    n = len(jobs)
    codes, nmask = g.pack_planes(u8)
    d_out = torch.full((n * 7,), -777, dtype=torch.int32, device="cuda")
    d_st = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    ctx().align2_batch(sc, to_dev(jobs), n, to_dev(codes), to_dev(nmask), g.KSW_XSTART, int(jobs["tlen"].max()),
                       d_out, d_st, n_bases=len(u8))
    torch.cuda.synchronize()
    out, st = d_out.cpu().numpy().view(g.SWR_DT), d_st.cpu().numpy()
    assert (st[bad] == g.G3X_ERR_INVALID).all()
    assert (st[~bad] == 0).all()
    np.testing.assert_array_equal(out[~bad], want.astype(g.SWR_DT)[~bad])
