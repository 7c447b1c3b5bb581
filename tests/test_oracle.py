"""The CPU oracle (oracle/ksw_oracle.c) pinned against the reference's own code: the
committed golden vectors (generated from the reference's compiled ksw_extend2 and
mem_chain2aln lines) and, where oracle/_ref is built, fresh seeded jobs."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import golden_io, native as nat

REG_FIELDS = ["rb", "re", "qb", "qe", "score", "truesc", "w"]


@pytest.mark.parametrize("name", golden_io.job_sets())
def test_oracle_matches_golden_jobs(name):
    u8, jobs, score, ext = golden_io.load_jobs(name)
    out, cells, rows = nat.oracle_extend(jobs, u8, score)
    assert len(jobs) > 0
    bad = np.nonzero((out != ext).any(1))[0]
    assert bad.size == 0, f"{name}: first mismatching job {bad[:5]}"


@pytest.mark.parametrize("name", golden_io.seed_sets())
def test_oracle_seed_driver_matches_golden(name):
    u8, seeds, opt, reg = golden_io.load_seeds(name)
    out = nat.oracle_seeds(seeds, u8, opt)
    for f in REG_FIELDS:
        assert (out[f] == reg[f]).all(), f


def test_golden_covers_band_retry():
    u8, seeds, opt, reg = golden_io.load_seeds("cfg5_w5")
    out = nat.oracle_seeds(seeds, u8, opt)
    assert ((out["tries_left"] > 1) | (out["tries_right"] > 1)).sum() > 10
    assert (reg["w"] == 10).sum() > 10        # doubled band recorded in the region


def test_golden_covers_stale_reads():
    """The stale set holds jobs whose answer changes if stale buffer entries read as 0."""
    u8, jobs, score, ext = golden_io.load_jobs("stale")
    assert len(jobs) >= 10


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (reference tree absent)")
@pytest.mark.parametrize("kind,n,w", [(1, 20000, 100), (2, 10000, 100), (2, 5000, 7), (4, 40, 500)])
def test_oracle_matches_reference_fresh(kind, n, w):
    wl = g.synth(kind, n, seed=900 + kind + w, w=w)
    sc = g.default_score()
    a, _, _ = nat.oracle_extend(wl.jobs, wl.u8, sc)
    b = nat.ref_extend(wl.jobs, wl.u8, sc)
    assert (a == b).all()


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (reference tree absent)")
def test_seed_driver_matches_reference_fresh():
    sc = g.default_score()
    for w in (100, 6):
        wl = g.synth(2, 4000, seed=77 + w, w=w)
        opt = nat.opt_from_score(sc, w=w)
        a = nat.oracle_seeds(wl.seeds, wl.u8, opt)
        b = nat.ref_seeds(wl.seeds, wl.u8, opt)
        for f in REG_FIELDS:
            assert (a[f] == b[f]).all(), (w, f)


def test_band_clamp_integer_form():
    """(int)((double)(qlen*max + bonus - o)/e + 1.) clamped to >= 1 (ksw.cu:325-329) equals
    the integer form the kernels use: num >= 0 ? num/e + 1 : 1."""
    for e in (1, 2, 3, 7):
        for num in range(-300, 3000):
            ref = int(float(num) / e + 1.0)
            ref = ref if ref > 1 else 1
            mine = num // e + 1 if num >= 0 else 1
            mine = mine if mine > 1 else 1
            assert ref == mine, (num, e)


def test_oracle_cells_count_trip_count():
    """Cells = sum over executed rows of (end - beg); bounded by qlen * rows."""
    wl = g.synth(1, 2000, seed=5)
    out, cells, rows = nat.oracle_extend(wl.jobs, wl.u8, g.default_score())
    assert (cells <= wl.jobs["qlen"].astype(np.int64) * rows).all()
    assert (rows <= wl.jobs["tlen"]).all()
    assert cells.sum() > 0
