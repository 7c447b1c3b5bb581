"""The oracle's striped local alignment (g3o_ksw_align2 in oracle/ksw_oracle.c: ksw_align2,
ksw_qinit and ksw_i16 of bwa/src/ksw.cu:18-292) against the committed golden vectors of the
reference's own ksw_align2 (tests/golden/sw_*.npz, made by tests/golden/make_golden.py) and
against the compiled reference itself on fresh seeded windows.  Every kswr_t field is compared
(score, te, qe, score2, te2, tb, qb) under each flag set: plain, XSTART (start positions),
XSUBO (second-best score), XSTOP (stop at a score) and their combinations."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import golden_io
from tests import native as nat


@pytest.mark.parametrize("name", golden_io.sw_sets())
def test_oracle_sw_matches_golden(name):
    u8, jobs, score, xtras, out = golden_io.load_sw(name)
    cj = nat.cpu_jobs(jobs)
    for x, want in zip(xtras, out):
        got, _ = nat.oracle_sw(cj, u8, score, int(x))
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, f"xtra {int(x):#x}: jobs {bad[:5]}: {got[bad[:2]]} vs {want[bad[:2]]}"


def test_golden_sw_covers_the_paths():
    """The fixtures exercise second-best scores, start positions, early stops and ties."""
    u8, jobs, score, xtras, out = golden_io.load_sw("edge")
    by = dict(zip((int(x) for x in xtras), out))
    assert (by[nat.KSW_XSUBO]["score2"] > 0).any()
    assert (by[nat.KSW_XSTART]["tb"] > 0).any() and (by[nat.KSW_XSTART]["qb"] > 0).any()
    assert (by[nat.KSW_XSTOP | 15]["score"] < by[0]["score"]).any()
    assert (by[0]["score"] == 0).any() and (by[0]["te"] == -1).any()
    assert jobs["qlen"].max() == 256 and (jobs["tlen"] == 0).any()


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_sw_equals_reference(seed):
    cj, u8 = nat.sw_jobs(1500, 0xA11 + seed, rev_frac=0.25, related=0.6)
    sc = g.default_score()
    for x in (0, nat.KSW_XSTART, nat.KSW_XSTART | nat.KSW_XSUBO | 25, nat.KSW_XSUBO | 8, nat.KSW_XSTOP | 30):
        a, cells = nat.oracle_sw(cj, u8, sc, x)
        b = nat.ref_sw(cj, u8, sc, x)
        bad = np.nonzero(a != b)[0]
        assert bad.size == 0, f"xtra {x:#x}: jobs {bad[:5]}"
        rows = cj["tlen"] > 0                  # every pass enters at least one target row
        assert (cells[rows] >= cj["qlen"][rows]).all()


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
def test_oracle_sw_long_queries_equal_reference():
    """Queries of 257-500 bases (KSW_MAX_QLEN, bwa/src/ksw.h:11; beyond the GPU kernel's 256):
    the restatement still equals the reference, so the GPU limit is the kernel's, not the
    oracle's."""
    cj, u8 = nat.sw_jobs(300, 0xB16, flank=200, seed_len=(60, 120), max_q=500)
    assert cj["qlen"].max() > 256
    sc = g.default_score()
    for x in (0, nat.KSW_XSTART | nat.KSW_XSUBO | 30):
        a, _ = nat.oracle_sw(cj, u8, sc, x)
        b = nat.ref_sw(cj, u8, sc, x)
        assert np.array_equal(a, b), hex(x)


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
def test_oracle_sw_edge_of_int16_domain():
    """The GPU kernel's domain (queries up to 256 bases, any int8 matrix) keeps every cell at most
    127 * 256 + 127 < 2^15: the largest match score on identical 256-base sequences reaches
    127 * 256 exactly, and the reference's wrapping int16 adds agree with the oracle there."""
    rng = np.random.default_rng(0xE16)
    q = rng.integers(0, 4, 256).astype(np.uint8)
    u8 = np.concatenate([q, q])
    jobs = np.zeros(1, nat.CPU_JOB_DT)
    jobs["q_off"], jobs["t_off"], jobs["qlen"], jobs["tlen"] = 0, 256, 256, 256
    sc = g.default_score(a=127, b=1, o_del=1, e_del=1, o_ins=1, e_ins=1)
    for x in (0, nat.KSW_XSTART):
        a, _ = nat.oracle_sw(jobs, u8, sc, x)
        b = nat.ref_sw(jobs, u8, sc, x)
        assert np.array_equal(a, b) and int(a["score"][0]) == 127 * 256
