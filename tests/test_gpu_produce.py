"""The stage's inputs built on the GPU from the reference's own data: bwa's packed reference
to forward + reverse-complement planes, u8 reads to planes, and ExtendingPairGenerate's
per-seed windows (g3x_pair_generate).  Planes are compared word for word with the host packer,
windows and contig ids with the chain window rule restated in numpy, and a whole chain-level
call on GPU-built planes with the oracle."""
import numpy as np
import pytest

import g3sa_b200 as g
from g3sa_b200.chains import ALNREG_DT, pac_of, synth_chains
from tests import native as nat
from tests.gpu_util import ctx, to_dev

pytestmark = pytest.mark.gpu


def host_planes(u8, base, n_words, fill):
    codes = np.full(n_words * 2, fill, np.uint32)
    nmask = np.full(n_words, fill, np.uint32)
    assert g.lib().g3x_pack_codes(np.ascontiguousarray(u8).ctypes.data, len(u8), codes.ctypes.data,
                                  nmask.ctypes.data, base) == 0
    return codes, nmask


@pytest.mark.parametrize("base", [0, 37, 64, 1000])
def test_pac_to_planes_matches_host(base):
    import torch
    rng = np.random.default_rng(base)
    fwd = rng.integers(0, 4, 5003).astype(np.uint8)
    ref2 = np.concatenate([fwd, 3 - fwd[::-1]])
    n_words = (base + len(ref2)) // 32 + 3
    fill = 0xA5A5A5A5                                # the words' other bases must survive
    hc, hn = host_planes(ref2, base, n_words, fill)
    dc = torch.from_numpy(np.full(n_words * 2, fill, np.uint32).view(np.int32)).cuda()
    dn = torch.from_numpy(np.full(n_words, fill, np.uint32).view(np.int32)).cuda()
    g.pac_to_planes(to_dev(pac_of(fwd)), len(fwd), dc, dn, base)
    torch.cuda.synchronize()
    assert np.array_equal(dc.cpu().numpy().view(np.uint32), hc)
    assert np.array_equal(dn.cpu().numpy().view(np.uint32), hn)


@pytest.mark.parametrize("base", [0, 5, 96])
def test_pack_codes_device_matches_host(base):
    import torch
    rng = np.random.default_rng(7 + base)
    u8 = rng.integers(0, 6, 7777).astype(np.uint8)    # 4 and 5 are N
    n_words = (base + len(u8)) // 32 + 2
    fill = 0x3C3C3C3C
    hc, hn = host_planes(u8, base, n_words, fill)
    dc = torch.from_numpy(np.full(n_words * 2, fill, np.uint32).view(np.int32)).cuda()
    dn = torch.from_numpy(np.full(n_words, fill, np.uint32).view(np.int32)).cuda()
    g.pack_codes_device(to_dev(u8), len(u8), dc, dn, base)
    torch.cuda.synchronize()
    assert np.array_equal(dc.cpu().numpy().view(np.uint32), hc)
    assert np.array_equal(dn.cpu().numpy().view(np.uint32), hn)


def numpy_windows(wl, opt_np):
    """Per chain: (r0, r1, rid) by aux.cu:2134-2156 and bns_fetch_seq_gpu's clipping."""
    a, w = int(opt_np["a"][0]), int(opt_np["w"][0])
    od, ed, oi, ei = (int(opt_np[f][0]) for f in ("o_del", "e_del", "o_ins", "e_ins"))

    def gap(q):
        q = np.asarray(q, np.int64)
        ld = ((q * a - od) / ed + 1.0).astype(np.int64)
        li = ((q * a - oi) / ei + 1.0).astype(np.int64)
        return np.minimum(np.maximum(np.maximum(ld, li), 1), w << 1)

    lp = wl.l_pac
    lq_of = np.repeat(wl.reads["l_query"], wl.reads["n_chains"])
    out = {}
    for ci, ch in enumerate(wl.chains):
        if ch["n"] == 0:
            continue
        s = wl.seeds[ch["seed_beg"]:ch["seed_beg"] + ch["n"]]
        lq = int(lq_of[ci])
        tail = lq - s["qbeg"] - s["len"]
        r0 = max(int((s["rbeg"] - (s["qbeg"] + gap(s["qbeg"]))).min()), 0)
        r1 = min(int((s["rbeg"] + s["len"] + tail + gap(tail)).max()), 2 * lp)
        if r0 < lp < r1:
            if s["rbeg"][0] < lp:
                r1 = lp
            else:
                r0 = lp
        mid = int(s["rbeg"][0])
        rev = mid >= lp
        pf = 2 * lp - 1 - mid if rev else mid
        rid = int(np.searchsorted(wl.anns["offset"], pf, side="right") - 1)
        fb, fe = int(wl.anns["offset"][rid]), int(wl.anns["offset"][rid] + wl.anns["len"][rid])
        if rev:
            fb, fe = 2 * lp - fe, 2 * lp - fb
        out[ci] = (max(r0, fb), min(r1, fe), rid)
    return out


def test_pair_generate_windows_and_rid():
    import torch
    wl = synth_chains(800, seed=13, edge=0.4)
    opt = g.default_opt()
    opt_np = nat.opt_from_score(g.default_score())
    read_of = np.repeat(np.arange(wl.n_reads), wl.reads["n_chains"])
    recs = []
    for ci, ch in enumerate(wl.chains):
        for k in range(ch["n"]):
            recs.append((read_of[ci], ci, k))
    recs.append((wl.n_reads + 3, 0, 0))              # indexes outside the reads
    R = np.array(recs, np.int32).view(g.SEEDREC_DT).reshape(-1)
    n = len(R)
    d_out = torch.zeros(n * g.DSEED_DT.itemsize, dtype=torch.uint8, device="cuda")
    d_rid = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_st = torch.zeros(n, dtype=torch.int32, device="cuda")
    g.pair_generate(opt, wl.l_pac, wl.ref_off, to_dev(wl.anns), len(wl.anns), to_dev(wl.reads), wl.n_reads,
                    to_dev(wl.chains), len(wl.chains), to_dev(wl.seeds), len(wl.seeds), to_dev(R), n, d_out,
                    d_rid, d_st)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().view(g.DSEED_DT)
    rid, st = d_rid.cpu().numpy(), d_st.cpu().numpy()
    assert st[-1] == g.G3X_ERR_INVALID and (st[:-1] == 0).all()
    win = numpy_windows(wl, opt_np)
    for i in range(n - 1):
        r, ci, k = (int(x) for x in recs[i])
        r0, r1, cr = win[ci]
        s = wl.seeds[wl.chains[ci]["seed_beg"] + k]
        assert (out["rmax0"][i], out["rmax1"][i], rid[i]) == (r0, r1, cr)
        assert out["win_off"][i] == wl.ref_off + r0 and out["read_off"][i] == wl.reads["read_off"][r]
        assert (out["rbeg"][i], out["qbeg"][i], out["len"][i]) == (s["rbeg"], s["qbeg"], s["len"])


def test_chain2aln_on_gpu_built_planes():
    """Reference planes from the packed reference and read planes from the u8 reads, both
    built on the GPU, give the oracle's regions."""
    import torch
    wl = synth_chains(1500, seed=17, edge=0.2)
    L2 = 2 * wl.l_pac
    reads_u8 = wl.u8[L2:]
    n_words = (len(wl.u8) + 31) // 32 + 1
    dc = torch.zeros(n_words * 2, dtype=torch.int32, device="cuda")
    dn = torch.zeros(n_words, dtype=torch.int32, device="cuda")
    g.pac_to_planes(to_dev(pac_of(wl.u8[:wl.l_pac])), wl.l_pac, dc, dn, 0)
    g.pack_codes_device(to_dev(reads_u8), len(reads_u8), dc, dn, L2)
    opt_np = nat.opt_from_score(g.default_score())
    ref, rn, _ = nat.oracle_chains(wl, opt_np)
    ns = len(wl.seeds)
    regs = torch.zeros(ns * ALNREG_DT.itemsize, dtype=torch.uint8, device="cuda")
    nregs = torch.zeros(wl.n_reads, dtype=torch.int32, device="cuda")
    status = torch.zeros(wl.n_reads, dtype=torch.int32, device="cuda")
    ctx().chain2aln(g.default_opt(), wl.l_pac, wl.ref_off, to_dev(wl.anns), len(wl.anns), to_dev(wl.reads),
                    wl.n_reads, to_dev(wl.chains), len(wl.chains), to_dev(wl.seeds), ns, dc, dn, regs, nregs, status)
    torch.cuda.synchronize()
    assert (status.cpu().numpy() == 0).all()
    got = regs.cpu().numpy().view(ALNREG_DT)
    n = nregs.cpu().numpy()
    assert np.array_equal(n, rn)
    assert np.array_equal(nat.region_rows(got, n, wl.chains, wl.reads), nat.region_rows(ref, rn, wl.chains, wl.reads))
