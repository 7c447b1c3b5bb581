"""GPU parity: the sm_100a kernels through the C ABI against the golden vectors (computed by
the reference's own ksw_extend2) and against the oracle on fresh seeded workloads.  All six
outputs are compared bit-exactly; per-job cell counts equal the oracle's trip counts."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import golden_io, native as nat
from tests.gpu_util import run_batch

pytestmark = pytest.mark.gpu

R, P = g.KERNEL_ROLLING, g.KERNEL_ROWPAR
# (schedule, kernel, lanes, tile)
SCHEDULES = [(g.SCHED_PLAIN, R, 0, 0), (g.SCHED_SORTED, R, 8, 0), (g.SCHED_SORTED, R, 16, 0),
             (g.SCHED_SORTED, R, 32, 0), (g.SCHED_PLAIN, P, 0, 9)] + \
            [(g.SCHED_SORTED, P, l, t) for l in (4, 8, 16, 32) for t in (5, 9, 13)] + \
            [(g.SCHED_SORTED, g.KERNEL_LANE, 1, rf) for rf in (1, 8, 32)]
IDS = [f"{'plain' if s == 0 else 'pers'}-{ {R: 'roll', P: 'row', 3: 'lane'}[k]}-g{l}-c{t}" for s, k, l, t in SCHEDULES]


@pytest.mark.parametrize("sched,kernel,lanes,tile", SCHEDULES, ids=IDS)
@pytest.mark.parametrize("name", golden_io.job_sets())
def test_gpu_matches_golden(name, sched, kernel, lanes, tile):
    u8, jobs, score, ext = golden_io.load_jobs(name)
    if kernel == g.KERNEL_LANE and jobs["qlen"].max() > 1000:
        pytest.skip("the lane-per-job kernel holds each lane's query in shared memory (short queries)")
    out, status, cells = run_batch(u8, jobs, score, sched, lanes, tile=tile, kernel=kernel)
    assert (status == 0).all(), np.unique(status)
    bad = np.nonzero((out != ext).any(1))[0]
    assert bad.size == 0, f"{name}: jobs {bad[:5]} got {out[bad[:3]]} want {ext[bad[:3]]}"


@pytest.mark.parametrize("sched,kernel,lanes,tile", SCHEDULES, ids=IDS)
@pytest.mark.parametrize("kind,n,w", [(1, 30000, 100), (2, 15000, 100), (4, 150, 100), (4, 150, 500)])
def test_gpu_matches_oracle_fresh(kind, n, w, sched, kernel, lanes, tile):
    if kernel == g.KERNEL_LANE and kind == 4:
        pytest.skip("the lane-per-job kernel holds each lane's query in shared memory (short queries)")
    wl = g.synth(kind, n, seed=0x6A5 + 100 * kind + w, w=w, unrelated=0.2 if kind == 2 else 0.0)
    sc = g.default_score()
    ref, rcells, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
    out, status, cells = run_batch(wl.u8, wl.jobs, sc, sched, lanes, tile=tile, kernel=kernel)
    assert (status == 0).all()
    bad = np.nonzero((out != ref).any(1))[0]
    assert bad.size == 0, f"jobs {bad[:5]}"
    assert (cells == rcells).all()


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
