"""GPU parity of the traceback stage's pair preparation (g3x_traceback_pairs:
FINALIZEALN_preprocessing2 of bwa/src/aux.cu:2698-2745 with the band cap of traceback_baseline)
against the oracle's restatement, itself pinned to the reference's own lines
(tests/test_tbpair_oracle.py), and of the whole stage on the GPU: chain-level regions
(g3x_chain2aln) -> pairs -> banded global alignment with CIGAR, NM and MD
(g3x_ksw_global2_batch), against the oracle's chain level and global alignment."""
import numpy as np
import pytest

import g3sa_b200 as g
from g3sa_b200.chains import ALNREG_DT, synth_chains
from tests import native as nat
from tests.gpu_util import ctx, to_dev
from tests.test_gpu_chain import run_chains
from tests.test_tbpair_oracle import edge_regions

pytestmark = pytest.mark.gpu


def gpu_pairs(wl, regs, recs, opt):
    import torch
    n = len(recs)
    d_jobs = torch.zeros(max(n, 1) * g.JOB_DT.itemsize, dtype=torch.uint8, device="cuda")
    d_st = torch.full((max(n, 1),), 99, dtype=torch.int32, device="cuda")
    rec = np.zeros(n, g.ALNREC_DT)
    rec["read"], rec["reg"] = recs[:, 0], recs[:, 1]
    g.traceback_pairs(opt, wl.l_pac, wl.ref_off, to_dev(wl.reads), len(wl.reads), to_dev(regs), len(regs),
                      to_dev(rec), n, d_jobs, d_st)
    torch.cuda.synchronize()
    return d_jobs.cpu().numpy().view(g.JOB_DT)[:n], d_st.cpu().numpy()[:n]


def check_pairs(wl, regs, recs, opt, jobs, st):
    opt_cpu = nat.opt_from_score(g.default_score(), w=int(opt["w"][0]))
    q_off, qlen, tgt, tlen, w, rb = nat.oracle_tb_pairs(opt_cpu, wl.u8, wl.ref_off, wl.l_pac, wl.reads, regs,
                                                        recs, 4096)
    ok = st == 0
    assert ok.all(), np.unique(st)
    assert np.array_equal(jobs["q_off"], q_off) and np.array_equal(jobs["qlen"], qlen)
    assert np.array_equal(jobs["tlen"], tlen)
    assert np.array_equal(jobs["w"], np.minimum(w, 500))
    assert np.array_equal(jobs["flags"] == g.JOB_MDRC, rb >= wl.l_pac)
    for k in range(len(jobs)):
        t0 = int(jobs["t_off"][k])
        assert np.array_equal(wl.u8[t0:t0 + tlen[k]], tgt[k, :tlen[k]]), k


@pytest.mark.parametrize("seed,edge", [(3, 0.15), (11, 0.4)])
def test_gpu_traceback_pairs_match_oracle(seed, edge):
    wl = synth_chains(2000, seed=seed, edge=edge)
    opt = g.default_opt(w=100)
    regs, nregs, _ = nat.oracle_chains(wl, nat.opt_from_score(g.default_score(), w=100))
    recs = nat.tb_records(wl, nregs)
    extra, erecs = edge_regions(wl, len(regs), 600, seed)
    allregs = np.concatenate([regs, extra])
    allrecs = np.concatenate([recs, erecs])
    jobs, st = gpu_pairs(wl, allregs, allrecs, opt)
    check_pairs(wl, allregs, allrecs, opt, jobs, st)
    assert (jobs["w"] > 0).any() and (jobs["w"] == 0).any() and (jobs["tlen"] == 0).any()
    assert (jobs["w"] == 500).any()                      # the band cap of traceback_baseline


def test_gpu_traceback_pairs_reject_bad_records():
    wl = synth_chains(50, seed=2)
    regs = np.zeros(4, ALNREG_DT)
    regs["rb"], regs["re"], regs["qb"], regs["qe"] = 10, 40, 5, 2   # qe < qb
    L2 = 2 * wl.l_pac                                              # a slice wholly past the reference
    regs[3]["rb"], regs[3]["re"], regs[3]["qb"], regs[3]["qe"] = L2 + 10, L2 + 50, 0, 10
    recs = np.array([[0, 0], [len(wl.reads), 1], [0, 7], [-1, 0], [0, 3]], np.int32)
    jobs, st = gpu_pairs(wl, regs, recs, g.default_opt())
    assert (st == g.G3X_ERR_INVALID).all()
    assert (jobs["qlen"] == 0).all() and (jobs["tlen"] == 0).all()


@pytest.mark.parametrize("seed", [5, 17])
def test_gpu_traceback_stage_end_to_end(seed):
    """Regions from the GPU chain level, pairs and global alignments with NM/MD on the GPU:
    every field equal to the oracle's chain level, pairs and ksw_global2 + NM/MD."""
    import torch
    wl = synth_chains(1500, seed=seed, edge=0.3)
    opt = g.default_opt(w=100)
    opt_cpu = nat.opt_from_score(g.default_score(), w=100)
    regs_o, nregs_o, _ = nat.oracle_chains(wl, opt_cpu)
    regs, nregs, status = run_chains(wl, opt)
    assert (status == 0).all() and np.array_equal(nregs, nregs_o)
    recs = nat.tb_records(wl, nregs)
    jobs, st = gpu_pairs(wl, regs, recs, opt)
    check_pairs(wl, regs_o, recs, opt, jobs, st)
    n = len(jobs)
    codes, nmask = wl.planes()
    stride, md_stride = int((jobs["qlen"].astype(int) + jobs["tlen"]).max()) + 2, 1024
    d_score = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_cig = torch.zeros(n * stride, dtype=torch.int32, device="cuda")
    d_nc = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_nm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_md = torch.zeros(n * md_stride, dtype=torch.uint8, device="cuda")
    d_st = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    ctx().global_batch(g.default_score(), to_dev(jobs), n, to_dev(codes), to_dev(nmask), int(jobs["qlen"].max()),
                       int(jobs["tlen"].max()), int(jobs["w"].max()), d_score, d_cig, stride, d_nc, d_st,
                       d_nm=d_nm, d_md=d_md, md_stride=md_stride)
    torch.cuda.synchronize()
    assert (d_st.cpu().numpy() == 0).all()
    cj = nat.cpu_jobs(jobs)
    s_o, c_o, n_o, _ = nat.oracle_global(cj, wl.u8, g.default_score(), stride)
    nm_o, md_o = nat.oracle_nm_md(cj, wl.u8, c_o, n_o, md_stride)
    cig = d_cig.cpu().numpy().view(np.uint32).reshape(n, stride)
    nc = d_nc.cpu().numpy()
    assert np.array_equal(d_score.cpu().numpy(), s_o) and np.array_equal(nc, n_o)
    assert all(np.array_equal(cig[k, :nc[k]], c_o[k, :n_o[k]]) for k in range(n))
    assert np.array_equal(d_nm.cpu().numpy(), nm_o)
    md = d_md.cpu().numpy().reshape(n, md_stride)
    assert [bytes(md[k]).split(b"\0")[0].decode() for k in range(n)] == md_o
    assert (jobs["flags"] == g.JOB_MDRC).any() and (nm_o > 0).any()
