"""GPU parity of the chain-level call (g3x_chain2aln, mem_chain2aln of bwa/src/aux.cu:178-315)
against the oracle's restatement, itself pinned to the reference's own mem_chain2aln
(tests/test_chain_oracle.py): every region field and every read's region count bit-exact,
through the length-sorted width classes and through the plain kernel."""
import numpy as np
import pytest

import g3sa_b200 as g
from g3sa_b200.chains import ALNREG_DT, synth_chains
from tests import native as nat
from tests.gpu_util import ctx, to_dev

pytestmark = pytest.mark.gpu


def run_chains(wl, opt, schedule=g.SCHED_SORTED, reads=None):
    import torch
    reads = wl.reads if reads is None else reads
    codes, nmask = wl.planes()
    d = {k: to_dev(v) for k, v in (("reads", reads), ("chains", wl.chains), ("seeds", wl.seeds),
                                   ("anns", wl.anns), ("codes", codes), ("nmask", nmask))}
    n_seeds = len(wl.seeds)
    regs = torch.zeros(max(n_seeds, 1) * ALNREG_DT.itemsize, dtype=torch.uint8, device="cuda")
    nregs = torch.full((len(reads),), -1, dtype=torch.int32, device="cuda")
    status = torch.full((len(reads),), 99, dtype=torch.int32, device="cuda")
    ctx().chain2aln(opt, wl.l_pac, wl.ref_off, d["anns"], len(wl.anns), d["reads"], len(reads),
                    d["chains"], len(wl.chains), d["seeds"], n_seeds, d["codes"], d["nmask"], regs,
                    nregs, status, schedule=schedule)
    torch.cuda.synchronize()
    return regs.cpu().numpy().view(ALNREG_DT), nregs.cpu().numpy(), status.cpu().numpy()


@pytest.mark.parametrize("schedule", [g.SCHED_SORTED, g.SCHED_PLAIN])
@pytest.mark.parametrize("seed,w,edge", [(3, 100, 0.15), (11, 50, 0.3)])
def test_gpu_chain2aln_matches_oracle(seed, w, edge, schedule):
    wl = synth_chains(3000, seed=seed, edge=edge)
    sc = g.default_score()
    opt_cpu = nat.opt_from_score(sc, w=w)
    opt = g.default_opt(w=w)
    ref, rn, _ = nat.oracle_chains(wl, opt_cpu)
    regs, nregs, status = run_chains(wl, opt, schedule)
    assert (status == 0).all(), np.unique(status)
    assert np.array_equal(nregs, rn)
    a = nat.region_rows(regs, nregs, wl.chains, wl.reads)
    b = nat.region_rows(ref, rn, wl.chains, wl.reads)
    bad = np.nonzero(a != b)[0]
    assert bad.size == 0, f"{bad.size} regions differ, first {a[bad[:2]]} vs {b[bad[:2]]}"


def test_gpu_chain2aln_rejects_bad_records_per_read():
    """A read whose chain range runs past the chain array gets G3X_ERR_INVALID and no
    regions; the other reads are unaffected."""
    wl = synth_chains(400, seed=21)
    opt_cpu = nat.opt_from_score(g.default_score())
    ref, rn, _ = nat.oracle_chains(wl, opt_cpu)
    reads = wl.reads.copy()
    bad = 7
    reads["n_chains"][bad] = len(wl.chains) + 5
    regs, nregs, status = run_chains(wl, g.default_opt(), reads=reads)
    assert status[bad] == g.G3X_ERR_INVALID and nregs[bad] == 0
    keep = np.ones(len(reads), bool)
    keep[bad] = False
    assert (status[keep] == 0).all()
    assert np.array_equal(nregs[keep], rn[keep])


def test_gpu_chain2aln_empty_chains():
    """Reads without chains and chains without seeds give no regions."""
    wl = synth_chains(200, seed=4)
    reads = wl.reads.copy()
    reads["n_chains"][::5] = 0
    chains = wl.chains
    wl2 = synth_chains(200, seed=4)
    wl2.reads = reads
    opt_cpu = nat.opt_from_score(g.default_score())
    ref, rn, _ = nat.oracle_chains(wl2, opt_cpu)
    regs, nregs, status = run_chains(wl2, g.default_opt())
    assert (status == 0).all()
    assert (nregs[::5] == 0).all()
    assert np.array_equal(nregs, rn)
    assert np.array_equal(nat.region_rows(regs, nregs, chains, reads), nat.region_rows(ref, rn, chains, reads))
