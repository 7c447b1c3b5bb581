"""The oracle's pair preparation of the traceback stage (g3o_tb_pairs in oracle/ksw_oracle.c)
against the reference's own lines (FINALIZEALN_preprocessing2_kernel, bwa/src/aux.cu:2698-2737,
with infer_bw, aux.cu:506-513, and bns_get_seq_gpu, bwa/src/bntseq.cu:39-60, compiled by
oracle/build_ref.sh): query offset and length, the reference slice's bases and length, the band
width and rb, on the regions of chain-level calls and on hand-made regions (spanning the
forward/reverse boundary, reversed bounds, outside [0, 2 l_pac), equal lengths, any score)."""
import numpy as np
import pytest

import g3sa_b200 as g
from g3sa_b200.chains import ALNREG_DT, synth_chains
from tests import native as nat


def edge_regions(wl, first, n, seed):
    """n hand-made regions (indices first ..) with records on random reads."""
    rng = np.random.default_rng(seed)
    regs = np.zeros(n, ALNREG_DT)
    L2 = 2 * wl.l_pac
    for k in range(n):
        rb = int(rng.integers(-50, L2 + 50))
        ln = int(rng.integers(-30, 300))
        regs[k]["rb"], regs[k]["re"] = rb, rb + ln
        if k % 7 == 0:                                   # spans the forward/reverse boundary
            regs[k]["rb"], regs[k]["re"] = wl.l_pac - 20, wl.l_pac + 30
        if k % 11 == 5:                                  # far longer than the query: band > 500
            regs[k]["re"] = regs[k]["rb"] + int(rng.integers(1500, 3000))
        qb = int(rng.integers(0, 50))
        ql = ln if (k % 5 == 0 and ln > 0) else int(rng.integers(1, 200))   # equal lengths every fifth
        regs[k]["qb"], regs[k]["qe"] = qb, qb + ql
        regs[k]["score"] = int(rng.integers(-10, 200))
        lo, hi = sorted((int(regs[k]["rb"]), int(regs[k]["re"])))
        if hi < 0 or lo >= L2:         # a slice wholly outside [0, 2 l_pac): the reference asks its
            regs[k]["rb"], regs[k]["re"] = 0, 40   # arena for a negative size; not a region
    recs = np.stack([rng.integers(0, len(wl.reads), n), np.arange(first, first + n)], 1).astype(np.int32)
    return regs, recs


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
@pytest.mark.parametrize("seed,edge,w", [(3, 0.15, 100), (11, 0.4, 50)])
def test_oracle_tb_pairs_equal_reference(seed, edge, w):
    wl = synth_chains(1500, seed=seed, edge=edge)
    opt = nat.opt_from_score(g.default_score(), w=w)
    regs, nregs, _ = nat.oracle_chains(wl, opt)
    recs = nat.tb_records(wl, nregs)
    extra, erecs = edge_regions(wl, len(regs), 500, seed)
    allregs, allrecs = np.concatenate([regs, extra]), np.concatenate([recs, erecs])
    a = nat.oracle_tb_pairs(opt, wl.u8, wl.ref_off, wl.l_pac, wl.reads, allregs, allrecs, 4096)
    b = nat.ref_tb_pairs(opt, wl.u8, wl.ref_off, wl.l_pac, wl.reads, allregs, allrecs, 4096)
    for x, y, name in zip(a, b, ("q_off", "qlen", "tgt", "tlen", "w", "rb")):
        assert np.array_equal(x, y), name
    q_off, qlen, tgt, tlen, w, rb = a
    assert (w == 0).any() and (w > 0).any() and (tlen == 0).any() and (rb >= wl.l_pac).any()
    assert (w > 500).any()                               # the traceback stage caps these at 500


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
def test_oracle_tb_pairs_other_scoring():
    """Unequal insertion and deletion costs and a = 2: both infer_bw calls and both max-gap terms
    matter."""
    wl = synth_chains(600, seed=9, edge=0.2)
    opt = nat.opt_from_score(g.default_score(a=2, b=3, o_del=5, e_del=2, o_ins=4, e_ins=3), a=2, w=60)
    regs, nregs, _ = nat.oracle_chains(wl, opt)
    recs = nat.tb_records(wl, nregs)
    extra, erecs = edge_regions(wl, len(regs), 400, 9)
    allregs, allrecs = np.concatenate([regs, extra]), np.concatenate([recs, erecs])
    a = nat.oracle_tb_pairs(opt, wl.u8, wl.ref_off, wl.l_pac, wl.reads, allregs, allrecs, 4096)
    b = nat.ref_tb_pairs(opt, wl.u8, wl.ref_off, wl.l_pac, wl.reads, allregs, allrecs, 4096)
    for x, y, name in zip(a, b, ("q_off", "qlen", "tgt", "tlen", "w", "rb")):
        assert np.array_equal(x, y), name
