"""The oracle's mem_chain2aln (oracle/ksw_oracle.c) against the reference's own mem_chain2aln
(bwa/src/aux.cu:168-175, 178-315 and bwa/src/bntseq.cu:5, 7-87, compiled by
oracle/build_ref.sh) on seeded chain workloads: every region field and every read's region
count equal.  The workloads cover the paths of the function: containment skips, the overlap
rescue, windows clipped to contigs and to one strand, seeds at the read's ends."""
import numpy as np
import pytest

import g3sa_b200 as g
from g3sa_b200.chains import synth_chains
from tests import native as nat


def windows(wl, opt):
    """(r0, r1, crossed, clipped) per non-empty chain: the span of aux.cu:186-205 before and
    after the strand and contig clipping."""
    a, w = int(opt["a"][0]), int(opt["w"][0])
    od, ed, oi, ei = (int(opt[f][0]) for f in ("o_del", "e_del", "o_ins", "e_ins"))

    def gap(q):
        q = np.asarray(q, np.int64)
        ld = ((q * a - od) / ed + 1.0).astype(np.int64)
        li = ((q * a - oi) / ei + 1.0).astype(np.int64)
        return np.minimum(np.maximum(np.maximum(ld, li), 1), w << 1)

    L2 = 2 * wl.l_pac
    out = []
    lq_of = np.repeat(wl.reads["l_query"], wl.reads["n_chains"])
    for ci, ch in enumerate(wl.chains):
        if ch["n"] == 0:
            continue
        s = wl.seeds[ch["seed_beg"]:ch["seed_beg"] + ch["n"]]
        lq = int(lq_of[ci])
        tail = lq - s["qbeg"] - s["len"]
        r0 = max(int((s["rbeg"] - (s["qbeg"] + gap(s["qbeg"]))).min()), 0)
        r1 = min(int((s["rbeg"] + s["len"] + tail + gap(tail)).max()), L2)
        crossed = r0 < wl.l_pac < r1
        out.append((r0, r1, crossed))
    return out


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
@pytest.mark.parametrize("seed,w,edge", [(3, 100, 0.15), (11, 50, 0.3), (29, 100, 0.5)])
def test_oracle_chain2aln_equals_reference(seed, w, edge):
    wl = synth_chains(1500, seed=seed, edge=edge)
    opt = nat.opt_from_score(g.default_score(), w=w)
    regs, nregs, cells = nat.oracle_chains(wl, opt)
    rregs, rnregs = nat.ref_chains(wl, opt)
    assert np.array_equal(nregs, rnregs)
    a = nat.region_rows(regs, nregs, wl.chains, wl.reads)
    b = nat.region_rows(rregs, rnregs, wl.chains, wl.reads)
    assert np.array_equal(a, b)
    # the paths are exercised: skipped seeds, several regions per read, left- and right-less
    # seeds, windows across the strand boundary
    assert nregs.sum() < len(wl.seeds)
    assert (nregs > 1).sum() > 0
    assert (a["qb"] == 0).any() and (a["qe"] == wl.reads["l_query"].max()).any()
    if edge >= 0.3:
        assert any(c for _, _, c in windows(wl, opt))
    assert cells.sum() > 0


def test_chain_records_layout():
    from g3sa_b200 import chains as C
    assert C.CSEED_DT.itemsize == 24 and C.CHAIN_DT.itemsize == 16 and C.READ_DT.itemsize == 24
    assert C.ANN_DT.itemsize == 16 and C.ALNREG_DT.itemsize == 56


def test_synth_chains_layout():
    """A read's chains are contiguous, and their seeds one range (the API's contract)."""
    wl = synth_chains(300, seed=5)
    for r in wl.reads:
        b = r["chain_beg"]
        for c in range(1, r["n_chains"]):
            assert wl.chains[b + c]["seed_beg"] == wl.chains[b + c - 1]["seed_beg"] + wl.chains[b + c - 1]["n"]
    assert (wl.u8[:2 * wl.l_pac] < 4).all()
    fwd = wl.u8[:wl.l_pac]
    assert np.array_equal(wl.u8[wl.l_pac:2 * wl.l_pac], 3 - fwd[::-1])
