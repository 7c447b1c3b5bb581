"""Test-only bindings: the CPU oracle (oracle/), the reference's own ksw_extend2 compiled
from its source (oracle/_ref/), and the CPU model of the kernels' warp protocol
(libg3x_emu.so).  Only tests, __graft_entry__.smoke() and bench.py's CPU arm import this."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libg3x_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libksw_ref.so")
EMU_SO = os.path.join(ROOT, "g3sa_b200", "libg3x_emu.so")
EMU16_SO = os.path.join(ROOT, "g3sa_b200", "libg3x_emu16.so")

# g3o_job / RefJob (oracle/ksw_oracle.c, oracle/ref_wrap.cpp)
CPU_JOB_DT = np.dtype([("q_off", "<i8"), ("t_off", "<i8"), ("qlen", "<i4"), ("tlen", "<i4"),
                       ("h0", "<i4"), ("w", "<i4"), ("flags", "<i4"), ("pad_", "<i4")])
# g3o_score / RefScore
CPU_SCORE_DT = np.dtype([("mat", "i1", 25), ("pad_", "i1", 3), ("o_del", "<i4"), ("e_del", "<i4"),
                         ("o_ins", "<i4"), ("e_ins", "<i4"), ("zdrop", "<i4"), ("end_bonus", "<i4")])
CPU_OPT_DT = np.dtype([("a", "<i4"), ("o_del", "<i4"), ("e_del", "<i4"), ("o_ins", "<i4"),
                       ("e_ins", "<i4"), ("w", "<i4"), ("zdrop", "<i4"), ("pen_clip5", "<i4"),
                       ("pen_clip3", "<i4"), ("mat", "i1", 25), ("pad_", "i1", 3)])
CPU_REG_DT = np.dtype([("rb", "<i8"), ("re", "<i8"), ("qb", "<i4"), ("qe", "<i4"), ("score", "<i4"),
                       ("truesc", "<i4"), ("w", "<i4"), ("tries_left", "<i4"),
                       ("tries_right", "<i4"), ("pad_", "<i4"), ("cells", "<i8")])

_oracle = _ref = _emu = _emu16 = None


def build_oracle():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        _oracle = ctypes.CDLL(ORACLE_SO)
        _oracle.g3o_extend_batch.argtypes = [ctypes.c_void_p, ctypes.c_int64] + [ctypes.c_void_p] * 5 + [ctypes.c_int]
        _oracle.g3o_extend_seeds.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64, ctypes.c_void_p]
        _oracle.g3o_ksw_extend2.restype = ctypes.c_int
        P, I64 = ctypes.c_void_p, ctypes.c_int64
        _oracle.g3o_chain2aln_reads.argtypes = [P, P, I64, I64, P, ctypes.c_int, P, I64, P, P, P, P, P]
        _oracle.g3o_chain2aln_reads.restype = None
        _oracle.g3o_global_batch.argtypes = [P, I64, P, P, P, P, ctypes.c_int32, P, P]
        _oracle.g3o_global_batch.restype = None
        _oracle.g3o_nm_md_batch.argtypes = [P, I64, P, P, ctypes.c_int32, P, P, P, ctypes.c_int32]
        _oracle.g3o_nm_md_batch.restype = None
        _oracle.g3o_sw_batch.argtypes = [P, I64, P, P, ctypes.c_int, P, P]
        _oracle.g3o_sw_batch.restype = None
        _oracle.g3o_tb_pairs.argtypes = [P, P, I64, I64, P, P, P, I64, P, P, P, ctypes.c_int32, P, P, P]
        _oracle.g3o_tb_pairs.restype = None
        _oracle.g3o_flt_chained_seeds.argtypes = [P, ctypes.c_int, P, I64, I64, P, ctypes.c_int, P, I64, P, P, P, P]
        _oracle.g3o_flt_chained_seeds.restype = None
    return _oracle


def have_ref():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
        _ref.g3r_ksw_extend2_batch.argtypes = [ctypes.c_void_p, ctypes.c_int64] + [ctypes.c_void_p] * 3 + [ctypes.c_int]
        _ref.g3r_extend_seeds.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64, ctypes.c_void_p]
        P, I64 = ctypes.c_void_p, ctypes.c_int64
        _ref.g3r_chain2aln_reads.argtypes = [P, P, I64, I64, P, ctypes.c_int, P, I64, P, P, P, P]
        _ref.g3r_chain2aln_reads.restype = ctypes.c_int
        _ref.g3r_global_batch.argtypes = [P, I64, P, P, P, P, ctypes.c_int32, P]
        _ref.g3r_global_batch.restype = ctypes.c_int
        _ref.g3r_nm_md_batch.argtypes = [P, I64, P, P, ctypes.c_int32, P, P, P, ctypes.c_int32]
        _ref.g3r_nm_md_batch.restype = ctypes.c_int
        _ref.g3r_sw_batch.argtypes = [P, I64, P, P, ctypes.c_int, P]
        _ref.g3r_sw_batch.restype = ctypes.c_int
        _ref.g3r_tb_pairs.argtypes = [P, P, I64, I64, P, P, P, I64, P, P, P, ctypes.c_int32, P, P, P]
        _ref.g3r_tb_pairs.restype = ctypes.c_int
        _ref.g3r_flt_chained_seeds.argtypes = [P, ctypes.c_int, P, I64, I64, P, ctypes.c_int, P, I64, P, P]
        _ref.g3r_flt_chained_seeds.restype = ctypes.c_int
    return _ref


def emu():
    global _emu
    if _emu is None:
        _emu = ctypes.CDLL(EMU_SO)
        _emu.g3x_emu_extend_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32] + [ctypes.c_void_p] * 4
    return _emu


def emu16_extend(jobs, u8, score):
    """(ext[n,6], cells[n], status[n]) from the CPU model of the int16x2 lane kernel's per-lane
    logic (libg3x_emu16.so); status -3 (too long) for jobs outside its int16 fit."""
    global _emu16
    if _emu16 is None:
        _emu16 = ctypes.CDLL(EMU16_SO)
        _emu16.g3x_emu16_extend.argtypes = [ctypes.c_void_p, ctypes.c_int32] + [ctypes.c_void_p] * 5
    n = len(jobs)
    jobs = np.ascontiguousarray(jobs)
    u8 = np.ascontiguousarray(u8)
    score = np.ascontiguousarray(score)
    out = np.zeros((n, 6), np.int32)
    cells = np.zeros(n, np.int32)
    status = np.zeros(n, np.int32)
    rc = _emu16.g3x_emu16_extend(jobs.ctypes.data, n, u8.ctypes.data, score.ctypes.data, out.ctypes.data,
                                 cells.ctypes.data, status.ctypes.data)
    assert rc == 0
    return out, cells, status


def cpu_jobs(jobs):
    j = np.zeros(len(jobs), CPU_JOB_DT)
    for f in ("q_off", "t_off", "qlen", "tlen", "h0", "w", "flags"):
        j[f] = jobs[f]
    return j


def cpu_score(score):
    s = np.zeros(1, CPU_SCORE_DT)
    for f in ("mat", "o_del", "e_del", "o_ins", "e_ins", "zdrop", "end_bonus"):
        s[f] = score[f]
    return s


def oracle_extend(jobs, u8, score, threads=8):
    """(ext[n,6] int32, cells[n] int64, rows[n] int32) from the C restatement."""
    n = len(jobs)
    cj = cpu_jobs(jobs)
    cs = cpu_score(score)
    out = np.zeros((n, 6), np.int32)
    cells = np.zeros(n, np.int64)
    rows = np.zeros(n, np.int32)
    u8 = np.ascontiguousarray(u8)
    oracle().g3o_extend_batch(cj.ctypes.data, n, u8.ctypes.data, cs.ctypes.data, out.ctypes.data,
                              cells.ctypes.data, rows.ctypes.data, threads)
    return out, cells, rows


def ref_extend(jobs, u8, score, threads=8):
    """ext[n,6] from the reference's own ksw_extend2 (oracle/_ref)."""
    n = len(jobs)
    cj = cpu_jobs(jobs)
    cs = cpu_score(score)
    out = np.zeros((n, 6), np.int32)
    u8 = np.ascontiguousarray(u8)
    ref().g3r_ksw_extend2_batch(cj.ctypes.data, n, u8.ctypes.data, cs.ctypes.data, out.ctypes.data, threads)
    return out


def emu_extend(jobs, codes, nmask, score, G):
    n = len(jobs)
    out = np.zeros((n, 6), np.int32)
    status = np.zeros(n, np.int32)
    cells = np.zeros(n, np.int32)
    stats = np.zeros((n, 4), np.int64)
    jobs = np.ascontiguousarray(jobs)
    emu().g3x_emu_extend_batch(score.ctypes.data, jobs.ctypes.data, n, codes.ctypes.data,
                               nmask.ctypes.data, G, out.ctypes.data, status.ctypes.data,
                               cells.ctypes.data, stats.ctypes.data)
    return out, status, cells, stats


def opt_from_score(score, a=1, w=100, pen_clip5=5, pen_clip3=5):
    o = np.zeros(1, CPU_OPT_DT)
    o["a"], o["w"], o["pen_clip5"], o["pen_clip3"] = a, w, pen_clip5, pen_clip3
    for f in ("o_del", "e_del", "o_ins", "e_ins", "zdrop", "mat"):
        o[f] = score[f]
    return o


def oracle_seeds(seeds, u8, opt):
    out = np.zeros(len(seeds), CPU_REG_DT)
    oracle().g3o_extend_seeds(opt.ctypes.data, np.ascontiguousarray(u8).ctypes.data,
                              np.ascontiguousarray(seeds).ctypes.data, len(seeds), out.ctypes.data)
    return out


# RefOpt layout (oracle/ref_seed_head.inc mem_opt_t)
REF_OPT_DT = np.dtype([("a", "<i4"), ("b", "<i4"), ("o_del", "<i4"), ("e_del", "<i4"), ("o_ins", "<i4"),
                       ("e_ins", "<i4"), ("pen_clip5", "<i4"), ("pen_clip3", "<i4"), ("w", "<i4"),
                       ("zdrop", "<i4"), ("mat", "i1", 25), ("pad_", "i1", 3)])


def ref_seeds(seeds, u8, opt):
    """Seed-level outputs (CPU_REG_DT, first 7 fields) from the reference's own mem_chain2aln
    band-retry lines."""
    ro = np.zeros(1, REF_OPT_DT)
    for f in ("a", "o_del", "e_del", "o_ins", "e_ins", "pen_clip5", "pen_clip3", "w", "zdrop", "mat"):
        ro[f] = opt[f]
    out = np.zeros(len(seeds), CPU_REG_DT)
    ref().g3r_extend_seeds(ro.ctypes.data, np.ascontiguousarray(u8).ctypes.data,
                           np.ascontiguousarray(seeds).ctypes.data, len(seeds), out.ctypes.data)
    return out


def _chain_args(wl):
    u8 = np.ascontiguousarray(wl.u8)
    parts = [np.ascontiguousarray(x) for x in (wl.anns, wl.reads, wl.chains, wl.seeds)]
    return u8, parts


def oracle_chains(wl, opt):
    """(regions ALNREG_DT per seed slot, nregs per read, DP cells per read) from the C
    restatement of mem_chain2aln."""
    from g3sa_b200.chains import ALNREG_DT
    u8, (anns, reads, chains, seeds) = _chain_args(wl)
    regs = np.zeros(max(len(seeds), 1), ALNREG_DT)
    nregs = np.zeros(len(reads), np.int32)
    cells = np.zeros(len(reads), np.int64)
    oracle().g3o_chain2aln_reads(opt.ctypes.data, u8.ctypes.data, wl.ref_off, wl.l_pac,
                                 anns.ctypes.data, len(anns), reads.ctypes.data, len(reads),
                                 chains.ctypes.data, seeds.ctypes.data, regs.ctypes.data,
                                 nregs.ctypes.data, cells.ctypes.data)
    return regs, nregs, cells


def ref_chains(wl, opt):
    """(regions, nregs) from the reference's own mem_chain2aln (oracle/_ref)."""
    from g3sa_b200.chains import ALNREG_DT
    u8, (anns, reads, chains, seeds) = _chain_args(wl)
    ro = np.zeros(1, REF_OPT_DT)
    for f in ("a", "o_del", "e_del", "o_ins", "e_ins", "pen_clip5", "pen_clip3", "w", "zdrop", "mat"):
        ro[f] = opt[f]
    regs = np.zeros(max(len(seeds), 1), ALNREG_DT)
    nregs = np.zeros(len(reads), np.int32)
    ref().g3r_chain2aln_reads(ro.ctypes.data, u8.ctypes.data, wl.ref_off, wl.l_pac, anns.ctypes.data,
                              len(anns), reads.ctypes.data, len(reads), chains.ctypes.data,
                              seeds.ctypes.data, regs.ctypes.data, nregs.ctypes.data)
    return regs, nregs


def region_rows(regs, nregs, chains, reads):
    """The regions each read produced, as one array in read order."""
    out = []
    for r in range(len(reads)):
        if nregs[r]:
            b = int(chains[reads["chain_beg"][r]]["seed_beg"])
            out.append(regs[b:b + int(nregs[r])])
    return np.concatenate(out) if out else regs[:0]


NEG_HALF = -0x40000000 // 2


def global_jobs(n, seed, max_len=160, ws=(0, 1, 3, 5, 17, 50, 100), n_frac=0.1):
    """n (query, target) pairs for banded global alignment: targets are the queries with a few
    substitutions and 1-base indels; some queries carry N codes.  Returns (CPU_JOB_DT jobs,
    u8 codes)."""
    rng = np.random.default_rng(seed)
    jobs = np.zeros(n, CPU_JOB_DT)
    bufs, off = [], 0
    for k in range(n):
        ql = int(rng.integers(0, max_len))
        q = rng.integers(0, 5 if rng.random() < n_frac else 4, ql).astype(np.uint8)
        t = list(q)
        for _ in range(int(rng.integers(0, 6))):
            if not t:
                break
            p, u = int(rng.integers(0, len(t))), rng.random()
            if u < 0.5:
                t[p] = int(rng.integers(0, 4))
            elif u < 0.75:
                del t[p]
            else:
                t.insert(p, int(rng.integers(0, 4)))
        t = np.array(t, np.uint8)
        jobs[k]["q_off"], jobs[k]["t_off"] = off, off + len(q)
        bufs += [q, t]
        off += len(q) + len(t)
        jobs[k]["qlen"], jobs[k]["tlen"] = len(q), len(t)
        jobs[k]["w"] = int(rng.choice(ws))
    return jobs, (np.concatenate(bufs) if bufs else np.zeros(1, np.uint8))


def _global(fn, jobs, u8, score, stride, with_cells):
    n = len(jobs)
    sc = cpu_score(score)
    s = np.zeros(n, np.int32)
    c = np.zeros(max(n * stride, 1), np.uint32)
    nc = np.zeros(n, np.int32)
    args = [np.ascontiguousarray(jobs).ctypes.data, n, np.ascontiguousarray(u8).ctypes.data, sc.ctypes.data,
            s.ctypes.data, c.ctypes.data, stride, nc.ctypes.data]
    cells = np.zeros(n, np.int64)
    if with_cells:
        args.append(cells.ctypes.data)
    fn(*args)
    return s, c.reshape(n, stride) if n else c[:0].reshape(0, stride), nc, cells


def oracle_global(jobs, u8, score, stride):
    """(score, cigar [n, stride], n_cigar, cells) from the C restatement of ksw_global2."""
    return _global(oracle().g3o_global_batch, jobs, u8, score, stride, True)


def ref_global(jobs, u8, score, stride):
    """(score, cigar, n_cigar) from the reference's own ksw_global2."""
    return _global(ref().g3r_global_batch, jobs, u8, score, stride, False)[:3]


def _nm_md(fn, jobs, u8, cigar, n_cigar, md_stride):
    n = len(jobs)
    nm = np.zeros(n, np.int32)
    md = np.zeros((max(n, 1), md_stride), np.uint8)
    cig = np.ascontiguousarray(cigar, np.uint32)
    fn(np.ascontiguousarray(jobs).ctypes.data, n, np.ascontiguousarray(u8).ctypes.data, cig.ctypes.data,
       cig.shape[1], np.ascontiguousarray(n_cigar, np.int32).ctypes.data, nm.ctypes.data, md.ctypes.data, md_stride)
    return nm, [bytes(md[k]).split(b"\0")[0].decode() for k in range(n)]


def oracle_nm_md(jobs, u8, cigar, n_cigar, md_stride):
    """(NM, MD strings) from the C restatement of the traceback stage's NM/MD block."""
    return _nm_md(oracle().g3o_nm_md_batch, jobs, u8, cigar, n_cigar, md_stride)


def ref_nm_md(jobs, u8, cigar, n_cigar, md_stride):
    """(NM, MD strings) from the reference's own NM/MD block (aux.cu:2830-2861)."""
    return _nm_md(ref().g3r_nm_md_batch, jobs, u8, cigar, n_cigar, md_stride)


# kswr_t (bwa/src/ksw.h:24-29) == g3o_swr == g3x_swr_t
SWR_DT = np.dtype([("score", "<i4"), ("te", "<i4"), ("qe", "<i4"), ("score2", "<i4"), ("te2", "<i4"),
                   ("tb", "<i4"), ("qb", "<i4")])
KSW_XSTOP, KSW_XSUBO, KSW_XSTART = 0x20000, 0x40000, 0x80000


def _mutate(rng, seq, div):
    """seq with substitutions, 1-3 base insertions and deletions at rate div."""
    out = []
    for b in seq:
        u = rng.random()
        if u < div * 0.7:
            out.append(int(rng.integers(0, 4)))
        elif u < div * 0.85:
            continue
        elif u < div:
            out.append(int(b))
            out.extend(int(x) for x in rng.integers(0, 4, int(rng.integers(1, 4))))
        else:
            out.append(int(b))
    return np.array(out, np.uint8)


def sw_jobs(n, seed, flank=50, seed_len=(19, 60), related=0.5, n_frac=0.05, rev_frac=0.0, max_q=199):
    """n seed-window pairs as mem_seed_sw cuts them (aux.cu:117-143): a seed of seed_len bases
    with up to `flank` bases either side on the read (the query) and on the reference (the
    target); the flanks agree with divergence U[0, 10%] for a `related` fraction of the pairs
    and are unrelated otherwise; some queries carry N codes.  Query and target stay below
    max_q + 1 bases.  A `rev_frac` fraction of the jobs has both sequences stored backwards
    (flags 1 | 2).  Returns (CPU_JOB_DT jobs, u8 codes)."""
    rng = np.random.default_rng(seed)
    jobs = np.zeros(n, CPU_JOB_DT)
    bufs, off = [], 0
    for k in range(n):
        L = int(rng.integers(seed_len[0], seed_len[1]))
        core = rng.integers(0, 4, L).astype(np.uint8)
        a, b = int(rng.integers(0, flank + 1)), int(rng.integers(0, flank + 1))
        ql, qr = rng.integers(0, 4, a).astype(np.uint8), rng.integers(0, 4, b).astype(np.uint8)
        q = np.concatenate([ql, core, qr])
        if rng.random() < related:
            div = rng.random() * 0.1
            tl, tr = _mutate(rng, ql, div), _mutate(rng, qr, div)
        else:
            tl = rng.integers(0, 4, int(rng.integers(0, flank + 1))).astype(np.uint8)
            tr = rng.integers(0, 4, int(rng.integers(0, flank + 1))).astype(np.uint8)
        t = np.concatenate([tl, _mutate(rng, core, 0.02), tr])
        q, t = q[:max_q], t[:max_q]
        if rng.random() < n_frac and len(q):
            q[rng.integers(0, len(q), int(rng.integers(1, 4)))] = 4
        flags = 3 if rng.random() < rev_frac else 0
        if flags:
            q, t = q[::-1].copy(), t[::-1].copy()
        jobs[k]["q_off"], jobs[k]["t_off"] = off, off + len(q)
        jobs[k]["qlen"], jobs[k]["tlen"], jobs[k]["flags"] = len(q), len(t), flags
        bufs += [q, t]
        off += len(q) + len(t)
    return jobs, (np.concatenate(bufs) if bufs else np.zeros(1, np.uint8))


def _sw(fn, jobs, u8, score, xtra, with_cells):
    n = len(jobs)
    out = np.zeros(max(n, 1), SWR_DT)
    args = [np.ascontiguousarray(jobs).ctypes.data, n, np.ascontiguousarray(u8).ctypes.data,
            cpu_score(score).ctypes.data, int(xtra), out.ctypes.data]
    cells = np.zeros(max(n, 1), np.int64)
    if with_cells:
        args.append(cells.ctypes.data)
    fn(*args)
    return out[:n], cells[:n]


def oracle_sw(jobs, u8, score, xtra):
    """(kswr_t records, cells) from the C restatement of ksw_align2."""
    return _sw(oracle().g3o_sw_batch, jobs, u8, score, xtra, True)


def ref_sw(jobs, u8, score, xtra):
    """kswr_t records from the reference's own ksw_align2 (its trap line left out)."""
    return _sw(ref().g3r_sw_batch, jobs, u8, score, xtra, False)[0]


def _mutate_many(rng, seq, owner, rate, n_owner):
    """Vectorised _mutate over a concatenation: seq[k] belongs to sequence owner[k] and mutates
    at rate[k].  Returns (new concatenation, new length of each of the n_owner sequences)."""
    u = rng.random(len(seq))
    sub = u < rate * 0.7
    dele = (u >= rate * 0.7) & (u < rate * 0.85)
    ins = (u >= rate * 0.85) & (u < rate)
    s = seq.copy()
    s[sub] = rng.integers(0, 4, int(sub.sum()))
    extra = np.where(ins, rng.integers(1, 4, len(seq)), 0)
    counts = np.where(dele, 0, 1 + extra)
    out = np.repeat(s, counts)
    first = np.cumsum(counts) - counts                 # where each kept base lands
    is_ins = np.ones(len(out), bool)
    is_ins[first[~dele]] = False
    out[is_ins] = rng.integers(0, 4, int(is_ins.sum()))
    lens = np.bincount(owner, weights=counts, minlength=n_owner).astype(np.int64)
    return out.astype(np.uint8), lens


def sw_windows(n, seed, flank=50, seed_len=(19, 60), related=0.5, n_frac=0.05):
    """The shapes of sw_jobs, generated without a per-job loop (for large batches): seeds of
    seed_len bases with up to `flank` bases either side; related flanks with divergence
    U[0, 10%], unrelated ones random; the core with 2% divergence; some queries with N codes.
    Returns (CPU_JOB_DT jobs, u8 codes), query and target of a job adjacent."""
    rng = np.random.default_rng(seed)
    L = rng.integers(seed_len[0], seed_len[1], n)
    A, B = rng.integers(0, flank + 1, n), rng.integers(0, flank + 1, n)
    ql = A + L + B
    q = rng.integers(0, 4, int(ql.sum())).astype(np.uint8)
    qo = np.cumsum(ql) - ql
    owner = np.repeat(np.arange(n), ql)
    pos = np.arange(len(q)) - np.repeat(qo, ql)
    in_core = (pos >= np.repeat(A, ql)) & (pos < np.repeat(A + L, ql))
    rel = rng.random(n) < related
    div = rng.random(n) * 0.1
    rate = np.where(in_core, 0.02, np.repeat(div, ql))
    # unrelated jobs: their flanks are replaced by random bases of random length after mutation
    keep_src = in_core | np.repeat(rel, ql)
    t, tl = _mutate_many(rng, q[keep_src], owner[keep_src], rate[keep_src], n)
    ua, ub = rng.integers(0, flank + 1, n), rng.integers(0, flank + 1, n)
    ua, ub = np.where(rel, 0, ua), np.where(rel, 0, ub)
    total_t = tl + ua + ub
    tbuf = rng.integers(0, 4, int(total_t.sum())).astype(np.uint8)
    to = np.cumsum(total_t) - total_t
    src_o = np.cumsum(tl) - tl
    dst = np.repeat(to + ua - src_o, tl) + np.arange(len(t))
    tbuf[dst] = t
    nq = rng.random(n) < n_frac
    for k in np.nonzero(nq)[0][:]:
        hit = rng.integers(0, ql[k], int(rng.integers(1, 4)))
        q[qo[k] + hit] = 4
    total = ql + total_t
    base = np.cumsum(total) - total
    u8 = np.empty(int(total.sum()), np.uint8)
    u8[np.repeat(base - qo, ql) + np.arange(len(q))] = q
    u8[np.repeat(base + ql - to, total_t) + np.arange(len(tbuf))] = tbuf
    jobs = np.zeros(n, CPU_JOB_DT)
    jobs["q_off"], jobs["t_off"] = base, base + ql
    jobs["qlen"], jobs["tlen"] = ql, total_t
    return jobs, u8


TBOPT_DT = np.dtype([("a", "<i4"), ("o_del", "<i4"), ("e_del", "<i4"), ("o_ins", "<i4"), ("e_ins", "<i4")])


def tb_records(wl, nregs):
    """(read, region index) for every region a chain-level call wrote: read r's regions start at
    its first chain's first seed slot."""
    recs = []
    for r, rd in enumerate(wl.reads):
        if rd["n_chains"] == 0:
            continue
        beg = int(wl.chains[rd["chain_beg"]]["seed_beg"])
        recs += [(r, beg + i) for i in range(int(nregs[r]))]
    return np.array(recs, np.int32).reshape(-1, 2)


def _tb(fn, opt, u8, ref_off, l_pac, reads, regs, recs, tstride):
    n = len(recs)
    o = np.zeros(1, TBOPT_DT)
    for f in ("a", "o_del", "e_del", "o_ins", "e_ins"):
        o[f] = opt[f]
    q_off = np.zeros(max(n, 1), np.int64)
    qlen, tlen, w = (np.zeros(max(n, 1), np.int32) for _ in range(3))
    rb = np.zeros(max(n, 1), np.int64)
    tgt = np.zeros((max(n, 1), tstride), np.uint8)
    fn(o.ctypes.data, np.ascontiguousarray(u8).ctypes.data, int(ref_off), int(l_pac), np.ascontiguousarray(reads).ctypes.data,
       np.ascontiguousarray(regs).ctypes.data, np.ascontiguousarray(recs, np.int32).ctypes.data, n, q_off.ctypes.data,
       qlen.ctypes.data, tgt.ctypes.data, tstride, tlen.ctypes.data, w.ctypes.data, rb.ctypes.data)
    return q_off[:n], qlen[:n], tgt[:n], tlen[:n], w[:n], rb[:n]


def oracle_tb_pairs(opt, u8, ref_off, l_pac, reads, regs, recs, tstride):
    """(q_off, qlen, target bases [n, tstride], tlen, w, rb) from the C restatement of the
    traceback stage's pair preparation."""
    return _tb(oracle().g3o_tb_pairs, opt, u8, ref_off, l_pac, reads, regs, recs, tstride)


def ref_tb_pairs(opt, u8, ref_off, l_pac, reads, regs, recs, tstride):
    """The same from the reference's own FINALIZEALN_preprocessing2 lines (aux.cu:2698-2737)."""
    return _tb(ref().g3r_tb_pairs, opt, u8, ref_off, l_pac, reads, regs, recs, tstride)


def oracle_flt_seeds(wl, opt, min_chain_weight=0):
    """(chains, seeds, window scores, cells) after the C restatement of mem_flt_chained_seeds:
    copies of the workload's chain and seed arrays, changed as the reference changes them in
    place; window score -1 for seeds it skips, -2 for seeds of reads it leaves alone."""
    ch, sd = wl.chains.copy(), wl.seeds.copy()
    sw = np.full(max(len(sd), 1), -2, np.int32)
    cells = np.zeros(1, np.int64)
    oracle().g3o_flt_chained_seeds(opt.ctypes.data, int(min_chain_weight), wl.u8.ctypes.data, int(wl.ref_off),
                                   int(wl.l_pac), np.ascontiguousarray(wl.anns).ctypes.data, len(wl.anns),
                                   np.ascontiguousarray(wl.reads).ctypes.data, len(wl.reads), ch.ctypes.data,
                                   sd.ctypes.data, sw.ctypes.data, cells.ctypes.data)
    return ch, sd, sw[:len(sd)], int(cells[0])


def ref_flt_seeds(wl, opt, min_chain_weight=0):
    """(chains, seeds) after the reference's own mem_flt_chained_seeds (aux.cu:145-162)."""
    ch, sd = wl.chains.copy(), wl.seeds.copy()
    ref().g3r_flt_chained_seeds(opt.ctypes.data, int(min_chain_weight), wl.u8.ctypes.data, int(wl.ref_off),
                                int(wl.l_pac), np.ascontiguousarray(wl.anns).ctypes.data, len(wl.anns),
                                np.ascontiguousarray(wl.reads).ctypes.data, len(wl.reads), ch.ctypes.data,
                                sd.ctypes.data)
    return ch, sd
