"""The oracle's restatements of the rows around the extension against committed golden vectors
made by the reference's own compiled code (tests/golden/make_golden.py --rows): the chain level
(mem_chain2aln), banded global alignment with CIGAR, NM and MD (ksw_global2 and the traceback
stage's NM/MD block), the traceback stage's pair preparation (FINALIZEALN_preprocessing2) and
the seed filter of long reads (mem_flt_chained_seeds with mem_seed_sw).  These run wherever the
repository is, with or without the reference tree."""
import numpy as np
import pytest

from tests import golden_io
from tests import native as nat


@pytest.mark.parametrize("name", golden_io.row_sets("chains"))
def test_oracle_chains_match_golden(name):
    d = golden_io.load_rows("chains", name)
    wl = golden_io.workload(d)
    regs, nregs, _ = nat.oracle_chains(wl, d["opt"])
    assert np.array_equal(nregs, d["nregs"])
    assert np.array_equal(nat.region_rows(regs, nregs, wl.chains, wl.reads),
                          nat.region_rows(d["regs"], d["nregs"], wl.chains, wl.reads))


@pytest.mark.parametrize("name", golden_io.row_sets("global"))
def test_oracle_global_matches_golden(name):
    d = golden_io.load_rows("global", name)
    jobs, u8 = d["jobs"], d["u8"]
    stride = d["cigar"].shape[1]
    sc, cig, nc, _ = nat.oracle_global(jobs, u8, d["score"], stride)
    assert np.array_equal(sc, d["out_score"])
    # where no in-band alignment reaches the last cell the reference's backtrack reads direction
    # bytes it never wrote (its CIGAR is undefined; the oracle's is empty)
    defined = d["out_score"] > -(1 << 29)
    assert np.array_equal(nc[defined], d["n_cigar"][defined]) and (nc[~defined] == 0).all()
    assert (~defined).any()
    assert all(np.array_equal(cig[k, :nc[k]], d["cigar"][k, :nc[k]]) for k in np.nonzero(defined)[0])
    nm, md = nat.oracle_nm_md(jobs, u8, d["cigar"], d["n_cigar"], 4 * stride + 16)
    assert np.array_equal(nm[defined], d["nm"][defined])
    assert [md[k] for k in np.nonzero(defined)[0]] == [str(d["md"][k]) for k in np.nonzero(defined)[0]]


@pytest.mark.parametrize("name", golden_io.row_sets("tbpairs"))
def test_oracle_tb_pairs_match_golden(name):
    d = golden_io.load_rows("tbpairs", name)
    wl = golden_io.workload(d)
    q_off, qlen, tgt, tlen, w, rb = nat.oracle_tb_pairs(d["opt"], wl.u8, wl.ref_off, wl.l_pac, wl.reads, d["regs"],
                                                        d["recs"], 4096)
    for x, name_ in ((q_off, "q_off"), (qlen, "qlen"), (tlen, "tlen"), (w, "w"), (rb, "rb")):
        assert np.array_equal(x, d[name_]), name_
    tcat = np.concatenate([tgt[k, :tlen[k]] for k in range(len(tlen))])
    assert np.array_equal(tcat, d["tgt"])
    assert (w > 500).any() and (w == 0).any() and (tlen == 0).any()


@pytest.mark.parametrize("name", golden_io.row_sets("seedflt"))
def test_oracle_seed_filter_matches_golden(name):
    d = golden_io.load_rows("seedflt", name)
    wl = golden_io.workload(d)
    ch, sd, sw, _ = nat.oracle_flt_seeds(wl, d["opt"], int(d["mcw"]))
    assert np.array_equal(ch["n"], d["out_chains"]["n"])
    for c, c2 in zip(ch, d["out_chains"]):
        a, b = int(c["seed_beg"]), int(c["n"])
        assert sd[a:a + b].tobytes() == d["out_seeds"][a:a + b].tobytes()
    assert (sw >= 0).any() and (ch["n"] < wl.chains["n"]).any()
