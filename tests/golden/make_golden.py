"""Generates the golden vectors in tests/golden/ from the reference's own code.

Run in a checkout where the reference tree exists (oracle/build_ref.sh has built
oracle/_ref/libksw_ref.so from bwa/src/ksw.cu and bwa/src/aux.cu):

    python tests/golden/make_golden.py

Every expected output is computed by the reference's compiled ksw_extend2 (job sets) or by
its compiled mem_chain2aln band-retry lines (seed sets); the oracle restatement is checked
against these files by tests/test_oracle.py and the GPU kernels by tests/test_gpu_parity.py.
Inputs are seeded synthetic jobs (g3sa_b200.synth) plus hand-built edge cases.

Files:
    jobs_<name>.npz   u8 (one byte per base), jobs (JOB_DT), score (SCORE_DT), ext (n x 6)
    seeds_<name>.npz  u8, seeds (SEED_DT), opt (CPU_OPT_DT), reg (CPU_REG_DT)
    sw_<name>.npz     u8, jobs (JOB_DT), score, xtras (flag sets), out (flag sets x n kswr_t)
                      from the reference's own ksw_align2 (its trap line left out)

    chains_<name>.npz the chain workload (u8, l_pac, anns, reads, chains, seeds), opt, and the
                      reference's mem_chain2aln regions and counts
    global_<name>.npz jobs, u8, score and the reference's ksw_global2 score, CIGAR, NM and MD
    tbpairs_<name>.npz the chain workload, regions, records and the reference's pair preparation
    seedflt_<name>.npz the chain workload with long reads, opt, min chain weight, and the chains
                      and seeds after the reference's mem_flt_chained_seeds

`python tests/golden/make_golden.py --sw` rewrites the sw_ files only, `--rows` the chains_,
global_, tbpairs_ and seedflt_ files only.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import g3sa_b200 as g  # noqa: E402
from tests import native as nat  # noqa: E402


class JobBuilder:
    """Collects explicit (query, target, h0, w, flags) jobs into one u8 buffer."""

    def __init__(self):
        self.parts, self.jobs, self.off = [], [], 0

    def add(self, q, t, h0, w, flags=0):
        q = np.asarray(q, np.uint8)
        t = np.asarray(t, np.uint8)
        qo = self.off
        self.parts.append(q)
        self.off += len(q)
        to = self.off
        self.parts.append(t)
        self.off += len(t)
        self.jobs.append((qo, to, len(q), len(t), h0, w, flags))

    def build(self):
        jobs = np.array(self.jobs, dtype=g.JOB_DT)
        u8 = np.concatenate(self.parts) if self.parts else np.zeros(0, np.uint8)
        return u8, jobs


def edge_jobs(rng):
    b = JobBuilder()
    rnd = lambda n: rng.integers(0, 4, n).astype(np.uint8)  # noqa: E731
    # qlen = 1, several h0 and targets
    for h0 in (1, 5, 7, 8, 19, 60):
        for t in ([0], [1], [4], [0, 0, 0], list(rnd(30))):
            b.add([0], t, h0, 100)
    # tlen < qlen, tlen = 0, qlen = 0
    for ql, tl in ((50, 10), (30, 1), (20, 0), (0, 20), (0, 0), (1, 0)):
        q = rnd(ql)
        t = q[:tl].copy() if tl <= ql else np.concatenate([q, rnd(tl - ql)])
        b.add(q, t, 30, 100)
    # h0 <= oe_ins and h0 = 0
    for h0 in (0, 1, 6, 7):
        q = rnd(40)
        b.add(q, np.concatenate([q, rnd(20)]), h0, 100)
    # all-N query, N-rich target
    b.add(np.full(40, 4, np.uint8), rnd(60), 50, 100)
    q = rnd(40)
    t = q.copy()
    t[::3] = 4
    b.add(q, t, 50, 100)
    # unrelated target: immediate z-drop / m == 0
    for h0 in (19, 100, 150):
        b.add(rnd(120), rnd(220), h0, 100)
    # band widths: w > qlen, w = 0, 1, 2, negative
    for w in (1000, 0, 1, 2, -1, -5):
        q = rnd(60)
        b.add(q, np.concatenate([q, rnd(30)]), 40, w)
    # ties: two-letter alphabet, short
    for _ in range(60):
        ql, tl = rng.integers(1, 9), rng.integers(1, 9)
        b.add(rng.integers(0, 2, ql), rng.integers(0, 2, tl), int(rng.integers(1, 20)), int(rng.integers(1, 6)))
    # large h0, long query
    q = rnd(600)
    b.add(q, np.concatenate([q, rnd(200)]), 1000, 100)
    # maximum query length of the long-segment configuration
    q = rnd(5000)
    t = q.copy()
    t[rng.random(5000) < 0.005] = rnd(1)[0]
    b.add(q, np.concatenate([t, rnd(200)]), 150, 500)
    # reversed reads through the flags
    q = rnd(80)
    t = np.concatenate([rnd(20), q[::-1]])
    b.add(q, t, 40, 100, g.JOB_QREV | g.JOB_TREV)
    b.add(q, t[::-1].copy(), 40, 100, g.JOB_QREV)
    return b


def find_stale_sensitive(score, want=16, seed0=4242):
    """Jobs whose outputs change when the stale row-buffer entries (left over from older rows
    when the band grows by two columns, bwa/src/ksw.cu:388-391) are read as zero instead."""
    orc = nat.oracle()
    orc.g3o_stale_scan.argtypes = [ctypes.c_void_p, ctypes.c_int64] + [ctypes.c_void_p] * 4
    found = JobBuilder()
    k = 0
    for it in range(20):
        wl = g.synth(1, 200000, seed=seed0 + it, w=100, unrelated=0.2)
        cj, cs = nat.cpu_jobs(wl.jobs), nat.cpu_score(score)
        flags = np.zeros(wl.n, np.int32)
        stale = np.zeros(wl.n, np.int32)
        orc.g3o_stale_scan(cj.ctypes.data, wl.n, wl.u8.ctypes.data, cs.ctypes.data,
                           flags.ctypes.data, stale.ctypes.data)
        for idx in np.nonzero(flags)[0]:
            jb = wl.jobs[idx]
            q = wl.u8[jb["q_off"]:jb["q_off"] + jb["qlen"]]
            t = wl.u8[jb["t_off"]:jb["t_off"] + jb["tlen"]]
            found.add(q, t, int(jb["h0"]), int(jb["w"]))
            k += 1
        print(f"stale search: batch {it}, found {k}", flush=True)
        if k >= want:
            break
    return found


def save_jobs(name, u8, jobs, score):
    ext = nat.ref_extend(jobs, u8, score)
    np.savez_compressed(os.path.join(HERE, f"jobs_{name}.npz"), u8=u8, jobs=jobs, score=score, ext=ext)
    print(f"jobs_{name}: {len(jobs)} jobs, {len(u8)} bases")


def save_seeds(name, wl, opt):
    reg = nat.ref_seeds(wl.seeds, wl.u8, opt)
    np.savez_compressed(os.path.join(HERE, f"seeds_{name}.npz"), u8=wl.u8, seeds=wl.seeds, opt=opt, reg=reg)
    print(f"seeds_{name}: {len(wl.seeds)} seeds")


SW_XTRAS = (0, nat.KSW_XSTART, nat.KSW_XSUBO | 20, nat.KSW_XSTART | nat.KSW_XSUBO | 30, nat.KSW_XSTOP | 15,
            nat.KSW_XSUBO, nat.KSW_XSTART | nat.KSW_XSUBO | 400)


def sw_edge_jobs(rng):
    """Edge cases of the striped local alignment: one-base queries, empty and one-base targets,
    all-N queries, identical pairs, query lengths on the 8-lane segment boundaries up to 256,
    long targets, tandem repeats (ties for the end position), several copies of the query in
    one target (second-best scores), sequences stored backwards."""
    b = JobBuilder()
    rnd = lambda n: rng.integers(0, 4, n).astype(np.uint8)  # noqa: E731
    for t in ([], [0], [1], [4], list(rnd(30)), list(rnd(300))):
        b.add([0], t, 0, 0)
    b.add(rnd(5), [], 0, 0)
    b.add([4] * 20, rnd(60), 0, 0)
    b.add(rnd(40), [4] * 40, 0, 0)
    for ql in (100, 199, 256):
        q = rnd(ql)
        b.add(q, q, 0, 0)
    for ql in (7, 8, 9, 15, 16, 17, 63, 64, 65, 127, 128, 129, 200, 255, 256):
        q = rnd(ql)
        t = np.concatenate([rnd(int(rng.integers(0, 40))), nat._mutate(rng, q, 0.05), rnd(int(rng.integers(0, 40)))])
        b.add(q, t, 0, 0)
    q = rnd(150)
    b.add(q, np.concatenate([rnd(1200), q, rnd(1500)]), 0, 0)
    rep = np.tile(np.array([0, 1, 2, 3], np.uint8), 30)
    b.add(rep, np.tile(np.array([0, 1, 2, 3], np.uint8), 45), 0, 0)
    b.add(np.tile(np.array([2, 2, 1], np.uint8), 20), np.tile(np.array([2, 1], np.uint8), 50), 0, 0)
    for _ in range(6):
        q = rnd(int(rng.integers(20, 90)))
        parts = []
        for _c in range(int(rng.integers(2, 5))):
            parts += [rnd(int(rng.integers(5, 200))), nat._mutate(rng, q, rng.random() * 0.2)]
        b.add(q, np.concatenate(parts + [rnd(30)]), 0, 0)
    for _ in range(6):
        q = rnd(int(rng.integers(30, 180)))
        t = np.concatenate([rnd(20), nat._mutate(rng, q, 0.05), rnd(20)])
        b.add(q[::-1].copy(), t[::-1].copy(), 0, 0, flags=3)
        b.add(q[::-1].copy(), t, 0, 0, flags=1)
    return b


def save_sw(name, u8, jobs, score):
    cj = nat.cpu_jobs(jobs)
    out = np.stack([nat.ref_sw(cj, u8, score, x) for x in SW_XTRAS]) if len(jobs) else np.zeros((0,), nat.SWR_DT)
    np.savez_compressed(os.path.join(HERE, f"sw_{name}.npz"), u8=u8, jobs=jobs, score=score,
                        xtras=np.array(SW_XTRAS, np.int32), out=out)
    print(f"sw_{name}: {len(jobs)} jobs x {len(SW_XTRAS)} flag sets")


def sw_main(rng):
    sc = g.default_score()
    u8, jobs = sw_edge_jobs(rng).build()
    save_sw("edge", u8, jobs, sc)
    cj, u8 = nat.sw_jobs(400, 0x5EED, rev_frac=0.2)
    save_sw("seeds", u8, _gpu_jobs(cj), sc)
    sc2 = g.default_score(a=2, b=3, o_del=5, e_del=2, o_ins=4, e_ins=3)
    cj, u8 = nat.sw_jobs(300, 0x5EED + 1)
    save_sw("score2", u8, _gpu_jobs(cj), sc2)


def _gpu_jobs(cj):
    jobs = np.zeros(len(cj), g.JOB_DT)
    for f in ("q_off", "t_off", "qlen", "tlen", "flags"):
        jobs[f] = cj[f]
    return jobs


def _wl_arrays(wl):
    return dict(u8=wl.u8, l_pac=np.int64(wl.l_pac), anns=wl.anns, reads=wl.reads, chains=wl.chains, seeds=wl.seeds)


def save_chains(name, wl, opt):
    regs, nregs = nat.ref_chains(wl, opt)
    np.savez_compressed(os.path.join(HERE, f"chains_{name}.npz"), opt=opt, regs=regs, nregs=nregs, **_wl_arrays(wl))
    print(f"chains_{name}: {len(wl.reads)} reads, {int(nregs.sum())} regions")
    return regs, nregs


def save_global(name, jobs, u8, score):
    stride = int((jobs["qlen"] + jobs["tlen"]).max()) + 2
    sc, cig, nc = nat.ref_global(jobs, u8, score, stride)
    md_stride = 4 * stride + 16
    nm, md = nat.ref_nm_md(jobs, u8, cig, nc, md_stride)
    np.savez_compressed(os.path.join(HERE, f"global_{name}.npz"), jobs=jobs, u8=u8, score=score, out_score=sc,
                        cigar=cig, n_cigar=nc, nm=nm, md=np.array(md, dtype=object).astype(str))
    print(f"global_{name}: {len(jobs)} pairs")


def save_tbpairs(name, wl, opt, regs, recs):
    q_off, qlen, tgt, tlen, w, rb = nat.ref_tb_pairs(opt, wl.u8, wl.ref_off, wl.l_pac, wl.reads, regs, recs, 4096)
    tcat = np.concatenate([tgt[k, :tlen[k]] for k in range(len(recs))]) if len(recs) else np.zeros(0, np.uint8)
    np.savez_compressed(os.path.join(HERE, f"tbpairs_{name}.npz"), opt=opt, regs=regs, recs=recs, q_off=q_off,
                        qlen=qlen, tgt=tcat, tlen=tlen, w=w, rb=rb, **_wl_arrays(wl))
    print(f"tbpairs_{name}: {len(recs)} records")


def save_seedflt(name, wl, opt, mcw):
    ch, sd = nat.ref_flt_seeds(wl, opt, mcw)
    np.savez_compressed(os.path.join(HERE, f"seedflt_{name}.npz"), opt=opt, mcw=np.int32(mcw), out_chains=ch,
                        out_seeds=sd, **_wl_arrays(wl))
    print(f"seedflt_{name}: {len(wl.reads)} reads, {int(ch['n'].sum())} of {int(wl.chains['n'].sum())} seeds kept")


def rows_main():
    """Golden vectors of the rows around the extension: chain level, global alignment with
    NM/MD, traceback pairs, seed filter (small references so the files stay small)."""
    from g3sa_b200.chains import synth_chains
    from tests.test_tbpair_oracle import edge_regions
    sc = g.default_score()
    small = dict(n_contigs=4, contig_len=(6000, 16000))
    wl = synth_chains(300, seed=0x6C, edge=0.3, **small)
    opt = nat.opt_from_score(sc, w=100)
    regs, nregs = save_chains("edge", wl, opt)
    recs = nat.tb_records(wl, nregs)
    extra, erecs = edge_regions(wl, len(regs), 200, 0x6C)
    save_tbpairs("edge", wl, opt, np.concatenate([regs, extra]), np.concatenate([recs, erecs]))
    cj, u8 = nat.global_jobs(600, 0x61, max_len=160)
    save_global("mixed", cj, u8, sc)
    sc2 = g.default_score(a=2, b=3, o_del=5, e_del=2, o_ins=4, e_ins=3)
    cj, u8 = nat.global_jobs(300, 0x62, max_len=120, ws=(0, 2, 9, 30))
    save_global("score2", cj, u8, sc2)
    wl = synth_chains(80, seed=0x5F, read_lens=(100, 720, 750, 1000, 1500), div=0.03, edge=0.3, **small)
    save_seedflt("long", wl, opt, 0)
    save_seedflt("mcw", wl, opt, 25)


def main():
    if not nat.have_ref():
        sys.exit("oracle/_ref/libksw_ref.so missing: run sh oracle/build_ref.sh first")
    rng = np.random.default_rng(2025)
    sc = g.default_score()
    wl = g.synth(1, 1500, seed=0x6A5 + 1, w=100)
    save_jobs("cfg1", wl.u8, wl.jobs, sc)
    wl = g.synth(2, 800, seed=0x6A5 + 2, w=100, unrelated=0.2)
    save_jobs("cfg2", wl.u8, wl.jobs, sc)
    for w in (100, 500):
        wl = g.synth(4, 12, seed=0x6A5 + 4 + w, w=w)
        save_jobs(f"cfg4_w{w}", wl.u8, wl.jobs, sc)
    u8, jobs = edge_jobs(rng).build()
    save_jobs("edge", u8, jobs, sc)
    # a different scoring: a=2 b=3, gaps 5/2 (del) and 4/3 (ins), zdrop 40, end bonus 12
    sc2 = g.default_score(a=2, b=3, o_del=5, e_del=2, o_ins=4, e_ins=3, zdrop=40, end_bonus=12)
    wl = g.synth(1, 600, seed=0x6A5 + 7, w=50, a=2, o_del=5, e_del=2, o_ins=4, e_ins=3)
    save_jobs("score2", wl.u8, wl.jobs, sc2)
    sc3 = g.default_score(zdrop=0)  # z-drop disabled
    wl = g.synth(2, 300, seed=0x6A5 + 8, w=100)
    save_jobs("nozdrop", wl.u8, wl.jobs, sc3)
    u8, jobs = find_stale_sensitive(sc).build()
    save_jobs("stale", u8, jobs, sc)
    for w in (100, 5):
        wl = g.synth(2, 1500, seed=0x6A5 + 5 + w, w=w, unrelated=0.2)
        save_seeds(f"cfg5_w{w}", wl, nat.opt_from_score(sc, w=w))
    sw_main(np.random.default_rng(2026))
    rows_main()


if __name__ == "__main__":
    if "--sw" in sys.argv or "--rows" in sys.argv:
        if not nat.have_ref():
            sys.exit("oracle/_ref/libksw_ref.so missing: run sh oracle/build_ref.sh first")
        if "--sw" in sys.argv:
            sw_main(np.random.default_rng(2026))
        if "--rows" in sys.argv:
            rows_main()
    else:
        main()
