"""GPU parity: the sm_100a kernels through the C ABI against the golden vectors (computed by
the reference's own ksw_extend2) and against the oracle on fresh seeded workloads.  All six
outputs are compared bit-exactly; per-job cell counts equal the oracle's trip counts."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import golden_io, native as nat
from tests.gpu_util import run_batch

pytestmark = pytest.mark.gpu

R, P, LN, L16, L2, B = (g.KERNEL_ROLLING, g.KERNEL_ROWPAR, g.KERNEL_LANE, g.KERNEL_LANE16, g.KERNEL_LANE2,
                        g.KERNEL_BAND)
# (schedule, kernel, lanes, tile)
SCHEDULES = [(g.SCHED_PLAIN, R, 0, 0), (g.SCHED_SORTED, R, 8, 0), (g.SCHED_SORTED, R, 16, 0),
             (g.SCHED_SORTED, R, 32, 0), (g.SCHED_PLAIN, P, 0, 9)] + \
            [(g.SCHED_SORTED, P, l, t) for l in (4, 8, 16, 32) for t in (5, 9, 13)] + \
            [(g.SCHED_SORTED, LN, 1, rf) for rf in (1, 8, 32)] + \
            [(g.SCHED_SORTED, L16, 1, rf) for rf in (1, 8, 32)] + \
            [(g.SCHED_SORTED, L2, 1, rf) for rf in (1, 8, 32)] + \
            [(g.SCHED_SORTED, B, 32, 256), (g.SCHED_SORTED, B, 32, 1024), (g.SCHED_PLAIN, B, 32, 512)]
NAMES = {R: "roll", P: "row", LN: "lane", L16: "lane16", L2: "lane2", B: "band"}
IDS = [f"{'plain' if s == 0 else 'pers'}-{NAMES[k]}-g{l}-c{t}" for s, k, l, t in SCHEDULES]


def lane_fits(jobs, score, kernel):
    """Jobs a lane-per-job kernel takes (the others get G3X_ERR_TOO_LONG): h0 >= 0 and every H
    below 2^15 (int32 lane kernel), or below 2^15 >> k with 2^k >= 1 + max_score (int16x2)."""
    max_sc = int(score["mat"][0].max())
    mn = np.minimum(jobs["qlen"], jobs["tlen"]).astype(np.int64)
    hmax = jobs["h0"].astype(np.int64) + max(max_sc, 0) * mn
    ok = (jobs["h0"] >= 0) & (jobs["qlen"] < 65535)
    if kernel in (LN, L2):
        return ok & (hmax < 32768)
    k = 0
    while (1 << k) < 1 + max_sc and k < 15:
        k += 1
    oe_del, oe_ins = int(score["o_del"][0] + score["e_del"][0]), int(score["o_ins"][0] + score["e_ins"][0])
    small = oe_del < 16384 and oe_ins < 16384 and int(score["e_ins"][0]) <= 4095 and int(score["e_del"][0]) <= 4095
    return ok & ((hmax << k) < 32768) & small


def clamped_w(jobs, score):
    """The band width after the clamp of ksw.cu:321-329: min(w, the insertion and deletion
    limits (int)((qlen * max_score + end_bonus - o) / e + 1.), each at least 1)."""
    q = jobs["qlen"].astype(np.int64)
    max_sc = int(score["mat"][0].max())
    eb = int(score["end_bonus"][0])
    w = jobs["w"].astype(np.int64)
    for o, e in ((int(score["o_ins"][0]), int(score["e_ins"][0])), (int(score["o_del"][0]), int(score["e_del"][0]))):
        num = q * max_sc + eb - o
        w = np.minimum(w, np.maximum(np.where(num >= 0, num // e + 1, 1), 1))
    return w


def band_fits(jobs, score, window):
    """Jobs the band kernel takes: the band's 2w' + 2 entries fit the window and every H stays
    below 2^21 (h0 + qlen * max_score)."""
    max_sc = int(score["mat"][0].max())
    hmax = np.maximum(jobs["h0"].astype(np.int64), 0) + jobs["qlen"].astype(np.int64) * max_sc
    return (2 * clamped_w(jobs, score) + 2 <= window) & (hmax < (1 << 21))


def check_status(jobs, score, kernel, status, tile=0):
    """Mask of the jobs whose outputs are compared: all of them, except the jobs a lane-per-job
    kernel or the band kernel must reject (which must carry G3X_ERR_TOO_LONG)."""
    if kernel == B:
        fits = band_fits(jobs, score, tile or 1024)
        assert (status[~fits] == g.G3X_ERR_TOO_LONG).all()
        assert (status[fits] == 0).all(), np.unique(status[fits])
        return fits
    if kernel in (LN, L16, L2):
        fits = lane_fits(jobs, score, kernel)
        assert (status[~fits] == g.G3X_ERR_TOO_LONG).all()
        assert (status[fits] == 0).all(), np.unique(status[fits])
        assert fits.mean() > 0.5
        return fits
    assert (status == 0).all(), np.unique(status)
    return np.ones(len(jobs), bool)


@pytest.mark.parametrize("sched,kernel,lanes,tile", SCHEDULES, ids=IDS)
@pytest.mark.parametrize("name", golden_io.job_sets())
def test_gpu_matches_golden(name, sched, kernel, lanes, tile):
    u8, jobs, score, ext = golden_io.load_jobs(name)
    if kernel in (LN, L16, L2) and jobs["qlen"].max() > 1000:
        pytest.skip("the lane-per-job kernels hold each lane's query in shared memory (short queries)")
    out, status, cells = run_batch(u8, jobs, score, sched, lanes, tile=tile, kernel=kernel)
    keep = check_status(jobs, score, kernel, status, tile)
    bad = np.nonzero(((out != ext).any(1)) & keep)[0]
    assert bad.size == 0, f"{name}: jobs {bad[:5]} got {out[bad[:3]]} want {ext[bad[:3]]}"


@pytest.mark.parametrize("sched,kernel,lanes,tile", SCHEDULES, ids=IDS)
@pytest.mark.parametrize("kind,n,w", [(1, 30000, 100), (2, 15000, 100), (4, 150, 100), (4, 150, 500)])
def test_gpu_matches_oracle_fresh(kind, n, w, sched, kernel, lanes, tile):
    if kernel in (LN, L16, L2) and kind == 4:
        pytest.skip("the lane-per-job kernels hold each lane's query in shared memory (short queries)")
    wl = g.synth(kind, n, seed=0x6A5 + 100 * kind + w, w=w, unrelated=0.2 if kind == 2 else 0.0)
    sc = g.default_score()
    ref, rcells, rrows = nat.oracle_extend(wl.jobs, wl.u8, sc)
    out, status, cells, rows = run_batch(wl.u8, wl.jobs, sc, sched, lanes, tile=tile, kernel=kernel,
                                         with_rows=True)
    keep = check_status(wl.jobs, sc, kernel, status, tile)
    bad = np.nonzero(((out != ref).any(1)) & keep)[0]
    assert bad.size == 0, f"jobs {bad[:5]}"
    assert (cells[keep] == rcells[keep]).all()
    assert (rows[keep] == rrows[keep]).all()          # the row loop's trips (ksw.cu:346)


# Width classes on the lane-per-job kernels (int16x2 and int32) with the row-parallel kernel
# as the last class: the scheduler routes every job a lane class cannot hold to the last class.
LANE_TILES = [(20, 1, 2, 0, 1), (36, 1, 2, 0, 32), (72, 1, 0, 0, 8), (144, 1, 4, 0, 32),
              (288, 1, 4, 0, 8), (1 << 30, 32, 9, 0, 1)]


@pytest.mark.parametrize("name", golden_io.job_sets())
def test_gpu_lane_classes_route_every_job(name):
    import torch
    from tests.gpu_util import to_dev
    u8, jobs, score, ext = golden_io.load_jobs(name)
    ctx = g.Context(0)
    ctx.set_tiles(LANE_TILES)
    codes, nmask = g.pack_planes(u8)
    d_jobs, d_codes, d_nmask = to_dev(jobs), to_dev(codes), to_dev(nmask)
    n = len(jobs)
    out = torch.full((n, 6), -777, dtype=torch.int32, device="cuda")
    status = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    ctx.extend_batch(score, d_jobs, n, d_codes, d_nmask, out, status, int(jobs["qlen"].max()),
                     int(jobs["tlen"].max()), schedule=g.SCHED_SORTED)
    torch.cuda.synchronize()
    assert (status.cpu().numpy() == 0).all()
    np.testing.assert_array_equal(out.cpu().numpy(), ext)


def test_gpu_too_long_jobs_get_status():
    u8, jobs, score, ext = golden_io.load_jobs("cfg1")
    lim = 60
    out, status, cells = run_batch(u8, jobs, score, g.SCHED_PLAIN, max_qlen=lim)
    long_ = jobs["qlen"] > lim
    assert (status[long_] == g.G3X_ERR_TOO_LONG).all()
    assert (status[~long_] == 0).all()
    assert (out[~long_] == ext[~long_]).all()


def test_gpu_rejects_bad_scoring():
    u8, jobs, score, ext = golden_io.load_jobs("edge")
    for field, val in (("m", 4), ("e_del", 0), ("e_ins", -1)):
        bad = score.copy()
        bad[field] = val
        with pytest.raises(g.G3xError) as ei:
            run_batch(u8, jobs, bad)
        assert ei.value.code == g.G3X_ERR_SCORE


def test_gpu_lane_classes_route_jobs_beyond_16_bits():
    """Seed scores that leave the int16x2 range (17000), the 16-bit fields (40000) or are
    negative: the scheduler sends those jobs to the last class, and every output is exact."""
    import torch
    from tests.gpu_util import to_dev
    u8, jobs, score, _ = golden_io.load_jobs("cfg1")
    jobs = jobs.copy()
    jobs["h0"][0::7] = 17000
    jobs["h0"][3::11] = 40000
    jobs["h0"][5::13] = -5
    ref, _, _ = nat.oracle_extend(jobs, u8, score)
    ctx = g.Context(0)
    ctx.set_tiles(LANE_TILES)
    codes, nmask = g.pack_planes(u8)
    d_jobs, d_codes, d_nmask = to_dev(jobs), to_dev(codes), to_dev(nmask)
    n = len(jobs)
    out = torch.full((n, 6), -777, dtype=torch.int32, device="cuda")
    status = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    ctx.extend_batch(score, d_jobs, n, d_codes, d_nmask, out, status, int(jobs["qlen"].max()),
                     int(jobs["tlen"].max()), schedule=g.SCHED_SORTED)
    torch.cuda.synchronize()
    assert (status.cpu().numpy() == 0).all()
    np.testing.assert_array_equal(out.cpu().numpy(), ref)


# The ring form of the lane kernel (row buffer and query codes in rings of 224 columns, for
# bands of w <= 104) on long queries; w = 500 jobs do not fit the ring and go to the last class.
RING_TILES = [(1000, 1, 224, 0, 8), (3000, 1, 224, 0, 32), (6000, 1, 224, 0, 1), (1 << 30, 32, 9, 0, 1)]


@pytest.mark.parametrize("name", ["cfg4_w100", "cfg4_w500", "cfg1", "stale", "edge"])
def test_gpu_ring_classes_exact(name):
    import torch
    from tests.gpu_util import to_dev
    u8, jobs, score, ext = golden_io.load_jobs(name)
    ctx = g.Context(0)
    ctx.set_tiles([(max(64, int(jobs["qlen"].max()) // 2), 1, 224, 0, 8)] + RING_TILES[1:]
                  if name not in ("cfg4_w100", "cfg4_w500") else RING_TILES)
    codes, nmask = g.pack_planes(u8)
    d_jobs, d_codes, d_nmask = to_dev(jobs), to_dev(codes), to_dev(nmask)
    n = len(jobs)
    out = torch.full((n, 6), -777, dtype=torch.int32, device="cuda")
    status = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    ctx.extend_batch(score, d_jobs, n, d_codes, d_nmask, out, status, int(jobs["qlen"].max()),
                     int(jobs["tlen"].max()), schedule=g.SCHED_SORTED)
    torch.cuda.synchronize()
    assert (status.cpu().numpy() == 0).all()
    np.testing.assert_array_equal(out.cpu().numpy(), ext)


def test_gpu_ring_long_fresh():
    """Fresh long-segment jobs (qlen log-uniform 500-5,000, w = 100) through ring classes."""
    import torch
    from tests.gpu_util import to_dev
    wl = g.synth(4, 400, seed=0x41A6, w=100, unrelated=0.0)
    sc = g.default_score()
    ref, rcells, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
    ctx = g.Context(0)
    ctx.set_tiles(RING_TILES)
    codes, nmask = wl.planes()
    d_jobs, d_codes, d_nmask = to_dev(wl.jobs), to_dev(codes), to_dev(nmask)
    out = torch.full((wl.n, 6), -777, dtype=torch.int32, device="cuda")
    status = torch.full((wl.n,), 99, dtype=torch.int32, device="cuda")
    cells = torch.full((wl.n,), -1, dtype=torch.int32, device="cuda")
    ctx.extend_batch(sc, d_jobs, wl.n, d_codes, d_nmask, out, status, int(wl.jobs["qlen"].max()),
                     int(wl.jobs["tlen"].max()), schedule=g.SCHED_SORTED, d_cells=cells)
    torch.cuda.synchronize()
    assert (status.cpu().numpy() == 0).all()
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    assert (cells.cpu().numpy() == rcells).all()


def test_gpu_int32_only_classes():
    """g3x_set_int16(ctx, 0): the context's int16x2 classes turn int32, set_tiles refuses tile 2,
    the autotuner keeps to int32 kernels, and the outputs stay the oracle's (long segments at
    w = 100 and short jobs, which the int16x2 kernel would otherwise take)."""
    import torch
    from tests.gpu_util import to_dev
    ctx = g.Context(0)
    assert any(t[1] == 1 and t[2] == 2 for t in ctx.get_tiles())
    ctx.set_int16(False)
    assert not any(t[1] == 1 and t[2] == 2 for t in ctx.get_tiles())
    with pytest.raises(g.G3xError):
        ctx.set_tiles([(128, 1, 2, 0, 8), (1 << 30, 32, 9, 0, 1)])
    sc = g.default_score()
    for kind, n, w in ((4, 300, 100), (2, 4000, 100)):
        wl = g.synth(kind, n, seed=0x1632 + kind, w=w, unrelated=0.1)
        ref, rcells, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
        codes, nmask = wl.planes()
        d_jobs, d_codes, d_nmask = to_dev(wl.jobs), to_dev(codes), to_dev(nmask)
        mq, mt = int(wl.jobs["qlen"].max()), int(wl.jobs["tlen"].max())
        tiles = ctx.autotune(sc, d_jobs, wl.n, d_codes, d_nmask, mq, mt)
        assert not any(t[1] == 1 and t[2] == 2 for t in tiles), tiles
        out = torch.full((wl.n, 6), -777, dtype=torch.int32, device="cuda")
        status = torch.full((wl.n,), 99, dtype=torch.int32, device="cuda")
        cells = torch.full((wl.n,), -1, dtype=torch.int32, device="cuda")
        ctx.extend_batch(sc, d_jobs, wl.n, d_codes, d_nmask, out, status, mq, mt,
                         schedule=g.SCHED_SORTED, d_cells=cells)
        torch.cuda.synchronize()
        assert (status.cpu().numpy() == 0).all()
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
        assert (cells.cpu().numpy() == rcells).all()
