"""Chains of seeds for the chain-level extension (g3x_chain2aln, mem_chain2aln of
bwa/src/aux.cu:178-315): record layouts and a seeded synthetic workload.

The reference is one code sequence of 2*l_pac bases, the forward strand of every contig then
its reverse complement (position p >= l_pac is 3 - forward[2*l_pac - 1 - p], the strand
layout of bwa/src/bntseq.cu:39-60), stored in the same code buffer as the reads.  A read's
chains are contiguous in the chain array and run in that order; a chain's seeds are
contiguous in the seed array, and the seeds of a read's chains follow one another, so the
read's regions (at most one per seed) go to the seed slots of its first chain onwards.
"""
import numpy as np

CSEED_DT = np.dtype([("rbeg", "<i8"), ("qbeg", "<i4"), ("len", "<i4"), ("score", "<i4"),
                     ("pad_", "<i4")])                                      # mem_seed_t, 24 B
CHAIN_DT = np.dtype([("seed_beg", "<i4"), ("n", "<i4"), ("rid", "<i4"), ("frac_rep", "<f4")])
READ_DT = np.dtype([("read_off", "<i8"), ("l_query", "<i4"), ("chain_beg", "<i4"),
                    ("n_chains", "<i4"), ("pad_", "<i4")])                  # 24 B
ANN_DT = np.dtype([("offset", "<i8"), ("len", "<i4"), ("pad_", "<i4")])   # bntann1_t, 16 B
ALNREG_DT = np.dtype([("rb", "<i8"), ("re", "<i8"), ("qb", "<i4"), ("qe", "<i4"), ("rid", "<i4"),
                      ("score", "<i4"), ("truesc", "<i4"), ("w", "<i4"), ("seedcov", "<i4"),
                      ("seedlen0", "<i4"), ("frac_rep", "<f4"), ("pad_", "<i4")])   # 56 B


class ChainWorkload:
    """u8 codes (reference at ref_off = 0, then the reads), the contigs, reads, chains, seeds."""

    def __init__(self, u8, l_pac, anns, reads, chains, seeds):
        self.u8, self.l_pac, self.anns = u8, l_pac, anns
        self.reads, self.chains, self.seeds = reads, chains, seeds
        self.ref_off = 0
        self._planes = None

    @property
    def n_reads(self):
        return len(self.reads)

    def planes(self):
        if self._planes is None:
            from g3sa_b200 import pack_planes
            self._planes = pack_planes(self.u8)
        return self._planes


def _exact_runs(read, ref_seg, rpos, min_len):
    """Maximal runs of read positions that match the reference on one diagonal, as
    (start, length) with length >= min_len."""
    n = len(read)
    ok = np.zeros(n, bool)
    valid = rpos >= 0
    ok[valid] = read[valid] == ref_seg[rpos[valid]]
    # position i continues the run of i-1 when both match and sit on consecutive reference bases
    cont = np.zeros(n, bool)
    cont[1:] = ok[1:] & ok[:-1] & (rpos[1:] == rpos[:-1] + 1)
    starts = np.nonzero(ok & ~cont)[0]
    if starts.size == 0:
        return []
    # a run ends before the next position that does not continue it
    brk = np.nonzero(~cont)[0]
    idx = np.searchsorted(brk, starts, side="right")
    ends = np.where(idx < brk.size, brk[np.minimum(idx, brk.size - 1)], n)
    lens = ends - starts
    keep = lens >= min_len
    return list(zip(starts[keep].tolist(), lens[keep].tolist()))


def _sample_read(rng, ref2, p, seg_end, lq, d):
    """A read of up to lq bases from ref2[p:], with substitutions at rate d and 1-3 base
    insertions and deletions at 0.2% each; returns (read codes, reference offset of each read
    base from p or -1 for inserted bases, reference bases consumed)."""
    ne = lq + 16
    u = rng.random(ne)
    kind = np.where(u < 0.002, 1, np.where(u < 0.004, 2, 0))     # 0 base, 1 insertion, 2 deletion
    ln = np.where(kind == 0, 1, rng.integers(1, 4, ne))
    emit = np.where(kind == 2, 0, ln)
    adv = np.where(kind == 1, 0, ln)
    ref_at = np.concatenate([[0], np.cumsum(adv)[:-1]])          # reference offset of each event
    ev = np.repeat(np.arange(ne), emit)                           # event of each read base
    sub = np.arange(ev.size) - np.repeat(np.cumsum(emit) - emit, emit)   # index within the event
    rpos = np.where(kind[ev] == 1, -1, ref_at[ev] + sub)
    rpos = rpos[:lq]
    limit = seg_end - 1 - p
    if (rpos >= limit).any():                                     # stop at the segment's end
        cut = int(np.argmax(rpos >= limit))
        rpos = rpos[:cut]
    n = len(rpos)
    read = rng.integers(0, 4, n).astype(np.uint8)                 # inserted bases stay random
    m = rpos >= 0
    base = ref2[p + rpos[m]]
    flip = rng.random(int(m.sum())) < d
    base = np.where(flip, (base + rng.integers(1, 4, base.size)) & 3, base)
    read[m] = base
    used = int(rpos[m].max()) + 1 if m.any() else 0
    return read, rpos.astype(np.int64), used


def synth_chains(n_reads, seed=1, n_contigs=12, contig_len=(20000, 120000), a=1,
                 div=0.05, min_seed=19, spurious=0.6, edge=0.15, read_lens=None):
    """Reads sampled from a random reference (substitutions at up to `div`, small indels),
    each with its true chain (exact-match seeds along the read's alignment, some split into
    overlapping pieces) and, with probability `spurious`, one or two chains of short seeds at
    random loci.  A fraction `edge` of the reads lies within a read length of a contig end, so
    windows are clipped to contigs and strands.  Read lengths are 100/150/250 (0.4/0.4/0.2), or
    drawn uniformly from `read_lens`."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(contig_len[0], contig_len[1], n_contigs)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]])
    l_pac = int(lens.sum())
    fwd = rng.integers(0, 4, l_pac).astype(np.uint8)
    ref2 = np.concatenate([fwd, (3 - fwd[::-1]).astype(np.uint8)])
    anns = np.zeros(n_contigs, ANN_DT)
    anns["offset"], anns["len"] = offs, lens
    # contig segments of the 2*l_pac space: forward, then reverse (contig order reversed)
    seg_b = np.concatenate([offs, 2 * l_pac - (offs + lens)])
    seg_e = np.concatenate([offs + lens, 2 * l_pac - offs])
    seg_rid = np.concatenate([np.arange(n_contigs), np.arange(n_contigs)])

    read_chunks, reads, chains, seeds = [], [], [], []
    base = 2 * l_pac
    for r in range(n_reads):
        lq = int(rng.choice([100, 150, 250], p=[0.4, 0.4, 0.2])) if read_lens is None else int(rng.choice(read_lens))
        sg = int(rng.integers(0, len(seg_b)))
        span = lq + 8
        lo, hi = int(seg_b[sg]), int(seg_e[sg]) - span
        if rng.random() < edge:
            p = lo + int(rng.integers(0, 40)) if rng.random() < 0.5 else hi - int(rng.integers(0, 40))
        else:
            p = int(rng.integers(lo, hi))
        d = rng.random() * div
        read, rpos, k = _sample_read(rng, ref2, p, int(seg_e[sg]), lq, d)
        lq = len(read)
        seg = ref2[p:p + k + 1]
        rs = []
        for qb, ln in _exact_runs(read, seg, rpos, min_seed):
            rs.append((p + int(rpos[qb]), qb, ln))
            if ln >= 2 * min_seed and rng.random() < 0.5:    # an overlapping piece of the run
                cut = int(rng.integers(1, ln - min_seed + 1))
                rs.append((p + int(rpos[qb]) + cut, qb + cut, ln - cut))
        ch = []
        if rs:
            ch.append((sorted(rs), int(seg_rid[sg])))
        if rng.random() < spurious:
            for _ in range(int(rng.integers(1, 3))):
                sg2 = int(rng.integers(0, len(seg_b)))
                p2 = int(rng.integers(seg_b[sg2] + lq, seg_e[sg2] - 2 * lq))
                ss = []
                for _ in range(int(rng.integers(1, 4))):
                    ln = int(rng.integers(min_seed, min_seed + 8))
                    qb = int(rng.integers(0, lq - ln + 1))
                    ss.append((p2 + qb + int(rng.integers(-3, 4)), qb, ln))
                ch.append((sorted(ss), int(seg_rid[sg2])))
        if len(ch) > 1 and rng.random() < 0.3:
            ch = ch[::-1]
        reads.append((base, lq, len(chains), len(ch)))
        read_chunks.append(read)
        base += lq
        for ss, rid in ch:
            chains.append((len(seeds), len(ss), rid, float(rng.random())))
            for rb, qb, ln in ss:
                sc = ln * a - (int(rng.integers(0, 4)) if rng.random() < 0.3 else 0)
                seeds.append((rb, qb, ln, sc))
    u8 = np.concatenate([ref2] + read_chunks)
    R = np.zeros(len(reads), READ_DT)
    if reads:
        R["read_off"], R["l_query"], R["chain_beg"], R["n_chains"] = np.array(reads, np.int64).T
    C = np.zeros(len(chains), CHAIN_DT)
    if chains:
        c = np.array(chains, np.float64)
        C["seed_beg"], C["n"], C["rid"] = c[:, 0], c[:, 1], c[:, 2]
        C["frac_rep"] = c[:, 3].astype(np.float32)
    S = np.zeros(len(seeds), CSEED_DT)
    if seeds:
        s = np.array(seeds, np.int64)
        S["rbeg"], S["qbeg"], S["len"], S["score"] = s[:, 0], s[:, 1], s[:, 2], s[:, 3]
    return ChainWorkload(u8, l_pac, anns, R, C, S)


def pac_of(fwd):
    """bwa's packed reference of forward codes 0-3: base k in byte k >> 2, bits ((~k) & 3) << 1
    (bwa/src/bntseq.cu:4-5)."""
    fwd = np.asarray(fwd, np.uint8)
    k = np.arange(len(fwd), dtype=np.int64)
    pac = np.zeros(len(fwd) // 4 + 1, np.uint8)
    np.bitwise_or.at(pac, k >> 2, ((fwd & 3).astype(np.uint8) << ((~k & 3) << 1).astype(np.uint8)))
    return pac
