"""GPU parity of the batched striped local alignment (g3x_ksw_align2_batch: ksw_align2 with
ksw_qinit and ksw_i16, bwa/src/ksw.cu:18-292) against the reference's own ksw_align2 through
the committed golden vectors, and against the oracle's restatement (pinned to the same
reference by tests/test_sw_oracle.py) on fresh seeded windows: every kswr_t field bit-exact
under each flag set, in all three segment classes, with reversed sequences, a second scoring,
and the per-job rejections."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import golden_io
from tests import native as nat
from tests.gpu_util import ctx, to_dev

pytestmark = pytest.mark.gpu

XTRAS = (0, g.KSW_XSTART, g.KSW_XSUBO | 20, g.KSW_XSTART | g.KSW_XSUBO | 30, g.KSW_XSTOP | 15, g.KSW_XSUBO)


def gpu_jobs(cj):
    j = np.zeros(len(cj), g.JOB_DT)
    for f in ("q_off", "t_off", "qlen", "tlen", "flags"):
        j[f] = cj[f]
    return j


def run_sw(jobs, u8, score, xtra, max_tlen=None, stream=None):
    import torch
    n = len(jobs)
    codes, nmask = g.pack_planes(u8)
    d_out = torch.full((max(n, 1) * 7,), -777, dtype=torch.int32, device="cuda")
    d_st = torch.full((max(n, 1),), 99, dtype=torch.int32, device="cuda")
    mt = (int(jobs["tlen"].max()) if n else 0) if max_tlen is None else max_tlen
    ctx().align2_batch(score, to_dev(jobs), n, to_dev(codes), to_dev(nmask), xtra, mt, d_out, d_st, stream=stream)
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(g.SWR_DT)[:n], d_st.cpu().numpy()[:n]


@pytest.mark.parametrize("name", golden_io.sw_sets())
def test_gpu_sw_matches_golden(name):
    u8, jobs, score, xtras, out = golden_io.load_sw(name)
    for x, want in zip(xtras, out):
        got, st = run_sw(jobs, u8, score, int(x))
        assert (st == 0).all(), (hex(int(x)), np.unique(st))
        bad = np.nonzero(got != want.astype(g.SWR_DT))[0]
        assert bad.size == 0, f"xtra {int(x):#x}: jobs {bad[:5]}: {got[bad[:2]]} vs {want[bad[:2]]}"


@pytest.mark.parametrize("seed,flank,max_q", [(3, 50, 199), (4, 120, 256), (5, 10, 64)])
def test_gpu_sw_matches_oracle(seed, flank, max_q):
    """mem_seed_sw-shaped windows (and wider ones reaching the 256-base limit) in every class."""
    cj, u8 = nat.sw_jobs(6000, 0x5A + seed, flank=flank, rev_frac=0.2, max_q=max_q)
    sc = g.default_score()
    for x in XTRAS:
        want, _ = nat.oracle_sw(cj, u8, sc, x)
        got, st = run_sw(gpu_jobs(cj), u8, sc, x)
        assert (st == 0).all(), np.unique(st)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, f"xtra {x:#x}: jobs {bad[:5]}: {got[bad[:2]]} vs {want[bad[:2]]}"


def test_gpu_sw_mixed_lengths_and_rejections():
    """Query lengths 0..300 in one batch: lengths 1..256 exact against the oracle, 0 rejected as
    invalid, above 256 as too long; under XSUBO a target above max_tlen is too long."""
    rng = np.random.default_rng(77)
    n = 3000
    parts, jobs, off = [], np.zeros(n, g.JOB_DT), 0
    for k in range(n):
        ql = int(rng.integers(0, 301))
        q = rng.integers(0, 4, ql).astype(np.uint8)
        t = np.concatenate([rng.integers(0, 4, int(rng.integers(0, 50))).astype(np.uint8),
                            nat._mutate(rng, q, 0.05), rng.integers(0, 4, int(rng.integers(0, 50))).astype(np.uint8)])
        jobs[k]["q_off"], jobs[k]["t_off"], jobs[k]["qlen"], jobs[k]["tlen"] = off, off + ql, ql, len(t)
        parts += [q, t]
        off += ql + len(t)
    u8 = np.concatenate(parts)
    sc = g.default_score()
    ok = (jobs["qlen"] >= 1) & (jobs["qlen"] <= 256)
    cj = nat.cpu_jobs(jobs[ok])
    for x in (g.KSW_XSTART, g.KSW_XSUBO | 10):
        max_tlen = int(np.percentile(jobs["tlen"], 90)) if x & g.KSW_XSUBO else None
        got, st = run_sw(jobs, u8, sc, x, max_tlen=max_tlen)
        assert (st[jobs["qlen"] == 0] == g.G3X_ERR_INVALID).all()
        assert (st[jobs["qlen"] > 256] == g.G3X_ERR_TOO_LONG).all()
        keep = ok.copy()
        if max_tlen is not None:
            long_t = ok & (jobs["tlen"] > max_tlen)
            assert long_t.any() and (st[long_t] == g.G3X_ERR_TOO_LONG).all()
            keep &= ~long_t
        assert (st[keep] == 0).all()
        want, _ = nat.oracle_sw(cj, u8, sc, x)
        sub = np.nonzero(keep[ok])[0]
        bad = np.nonzero(got[keep] != want[sub])[0]
        assert bad.size == 0, f"xtra {x:#x}: {bad[:5]}"
        rej = ~ok
        assert (got[rej]["score"] == 0).all() and (got[rej]["te"] == -1).all()


def test_gpu_sw_rejects_bad_calls():
    import torch
    cj, u8 = nat.sw_jobs(10, 1)
    jobs = gpu_jobs(cj)
    with pytest.raises(g.G3xError):
        run_sw(jobs, u8, g.default_score(), g.KSW_XBYTE)
    neg = g.default_score(a=0, b=1)            # no positive score: XSUBO's ceil(score / max) undefined
    with pytest.raises(g.G3xError):
        run_sw(jobs, u8, neg, g.KSW_XSUBO | 5)
    got, st = run_sw(jobs[:0], u8, g.default_score(), 0)   # an empty batch is a no-op
    assert len(got) == 0
    torch.cuda.synchronize()


def test_gpu_sw_edge_of_int16_domain():
    """Cells up to 127 * 256 (+ one score) in int16 lanes: identical and mutated 256-base pairs
    under a = 127 equal the oracle, the identical ones at exactly 127 * 256."""
    rng = np.random.default_rng(0xE17)
    parts, rows, off = [], [], 0
    for k in range(64):
        q = rng.integers(0, 4, 256 - (k % 5)).astype(np.uint8)
        t = q.copy() if k % 2 == 0 else nat._mutate(rng, q, 0.03)[:256]
        rows.append((off, off + len(q), len(q), len(t)))
        parts += [q, t]
        off += len(q) + len(t)
    jobs = np.zeros(len(rows), g.JOB_DT)
    jobs["q_off"], jobs["t_off"], jobs["qlen"], jobs["tlen"] = np.array(rows).T
    u8 = np.concatenate(parts)
    sc = g.default_score(a=127, b=1, o_del=1, e_del=1, o_ins=1, e_ins=1)
    for x in (0, g.KSW_XSTART):
        want, _ = nat.oracle_sw(nat.cpu_jobs(jobs), u8, sc, x)
        got, st = run_sw(jobs, u8, sc, x)
        assert (st == 0).all()
        assert np.array_equal(got, want)
        assert int(got["score"][0]) == 127 * 256
