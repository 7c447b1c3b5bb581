"""The oracle's seed filter of long reads (g3o_flt_chained_seeds with g3o_seed_sw in
oracle/ksw_oracle.c) against the reference's own mem_flt_chained_seeds and mem_seed_sw
(bwa/src/aux.cu:117-162, with the window fetch of bwa/src/bntseq.cu:7-87 and its ksw_align2,
compiled by oracle/build_ref.sh): every chain's seed count and every kept seed equal, on reads
long enough for the filter to run and short enough to be left alone, with and without a minimum
chain weight, and with a second scoring."""
import numpy as np
import pytest

import g3sa_b200 as g
from g3sa_b200.chains import synth_chains
from tests import native as nat

LONG = (100, 150, 700, 720, 750, 800, 1000, 1500, 2000)


def kept(ch, sd):
    return [sd[c["seed_beg"]:c["seed_beg"] + c["n"]].tobytes() for c in ch]


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
@pytest.mark.parametrize("seed,mcw", [(4, 0), (5, 25), (6, 0)])
def test_oracle_flt_seeds_equal_reference(seed, mcw):
    wl = synth_chains(400, seed=seed, read_lens=LONG, div=0.03, edge=0.3)
    opt = nat.opt_from_score(g.default_score(), w=100)
    c1, s1, sw, cells = nat.oracle_flt_seeds(wl, opt, mcw)
    c2, s2 = nat.ref_flt_seeds(wl, opt, mcw)
    assert np.array_equal(c1["n"], c2["n"])
    assert kept(c1, s1) == kept(c2, s2)
    # the paths: windows aligned and kept or dropped, seeds without a window, reads left alone
    assert (sw >= 0).any() and (sw == -1).any() and (c1["n"] < wl.chains["n"]).any() and cells > 0
    if mcw == 0:
        assert (sw == -2).any()


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
def test_oracle_flt_seeds_other_scoring():
    wl = synth_chains(250, seed=8, read_lens=(900, 1200), div=0.04, edge=0.2, a=2)
    opt = nat.opt_from_score(g.default_score(a=2, b=3, o_del=5, e_del=2, o_ins=4, e_ins=3), a=2, w=60)
    c1, s1, _, _ = nat.oracle_flt_seeds(wl, opt, 0)
    c2, s2 = nat.ref_flt_seeds(wl, opt, 0)
    assert np.array_equal(c1["n"], c2["n"]) and kept(c1, s1) == kept(c2, s2)
