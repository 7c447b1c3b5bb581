"""GPU parity of the seed filter of long reads (g3x_flt_chained_seeds: mem_flt_chained_seeds
with mem_seed_sw, bwa/src/aux.cu:117-162) against the oracle's restatement, itself pinned to
the reference's own functions (tests/test_seedflt_oracle.py): every seed's window score, every
chain's seed count and every kept seed equal; reads with records outside their arrays are
rejected and left untouched."""
import numpy as np
import pytest

import g3sa_b200 as g
from g3sa_b200.chains import CHAIN_DT, CSEED_DT, synth_chains
from tests import native as nat
from tests.gpu_util import ctx, to_dev
from tests.test_seedflt_oracle import LONG, kept

pytestmark = pytest.mark.gpu


def run_flt(wl, opt, mcw, reads=None):
    import torch
    reads = wl.reads if reads is None else reads
    codes, nmask = wl.planes()
    d_ch, d_sd = to_dev(wl.chains), to_dev(wl.seeds)
    d_sw = torch.full((max(len(wl.seeds), 1),), -9, dtype=torch.int32, device="cuda")
    d_st = torch.full((len(reads),), 99, dtype=torch.int32, device="cuda")
    ctx().flt_chained_seeds(opt, mcw, wl.l_pac, wl.ref_off, to_dev(wl.anns), len(wl.anns), to_dev(reads), len(reads),
                            d_ch, len(wl.chains), d_sd, len(wl.seeds), to_dev(codes), to_dev(nmask), d_st,
                            d_sw_score=d_sw)
    torch.cuda.synchronize()
    return (d_ch.cpu().numpy().view(CHAIN_DT), d_sd.cpu().numpy().view(CSEED_DT), d_sw.cpu().numpy()[:len(wl.seeds)],
            d_st.cpu().numpy())


@pytest.mark.parametrize("seed,mcw", [(4, 0), (5, 25), (7, 0)])
def test_gpu_flt_seeds_match_oracle(seed, mcw):
    wl = synth_chains(600, seed=seed, read_lens=LONG, div=0.03, edge=0.3)
    opt = g.default_opt(w=100)
    c1, s1, sw1, _ = nat.oracle_flt_seeds(wl, nat.opt_from_score(g.default_score(), w=100), mcw)
    c2, s2, sw2, st = run_flt(wl, opt, mcw)
    assert (st == 0).all(), np.unique(st)
    bad = np.nonzero(sw1 != sw2)[0]
    assert bad.size == 0, f"{bad.size} window scores differ, first {bad[:5]}: {sw1[bad[:3]]} vs {sw2[bad[:3]]}"
    assert np.array_equal(c1["n"], c2["n"])
    assert kept(c1, s1) == kept(c2, s2)


def test_gpu_flt_seeds_rejects_bad_reads():
    wl = synth_chains(120, seed=9, read_lens=(1000,), div=0.03)
    reads = wl.reads.copy()
    bad = 5
    reads["n_chains"][bad] = len(wl.chains) + 3
    c1, s1, _, _ = nat.oracle_flt_seeds(wl, nat.opt_from_score(g.default_score()), 0)
    c2, s2, sw2, st = run_flt(wl, g.default_opt(), 0, reads=reads)
    assert st[bad] == g.G3X_ERR_INVALID and (np.delete(st, bad) == 0).all()
    mine = slice(wl.reads["chain_beg"][bad], wl.reads["chain_beg"][bad] + wl.reads["n_chains"][bad])
    assert np.array_equal(c2["n"][mine], wl.chains["n"][mine])        # untouched
    keep = np.ones(len(wl.chains), bool)
    keep[mine] = False
    assert np.array_equal(c1["n"][keep], c2["n"][keep])
