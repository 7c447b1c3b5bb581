"""GPU parity of the batched banded global alignment (g3x_ksw_global2_batch, ksw_global2 of
bwa/src/ksw.cu:706-809) against the oracle's restatement, itself pinned to the reference's
own ksw_global2 (tests/test_global_oracle.py): scores and CIGARs bit-exact, empty CIGARs where
no in-band alignment reaches the last cell, reversed reads, and the job limits."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import native as nat
from tests.gpu_util import ctx, to_dev

pytestmark = pytest.mark.gpu


def gpu_jobs(cj, flags=0):
    j = np.zeros(len(cj), g.JOB_DT)
    j["q_off"], j["t_off"] = cj["q_off"], cj["t_off"]
    j["qlen"], j["tlen"], j["w"] = cj["qlen"], cj["tlen"], cj["w"]
    j["flags"] = flags
    return j


def run_global(jobs, u8, stride, max_qlen=None, max_tlen=None, max_w=None):
    import torch
    n = len(jobs)
    codes, nmask = g.pack_planes(u8)
    d_score = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_cig = torch.zeros(n * stride, dtype=torch.int32, device="cuda")
    d_nc = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_st = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    mq = int(jobs["qlen"].max()) if max_qlen is None else max_qlen
    mt = int(jobs["tlen"].max()) if max_tlen is None else max_tlen
    mw = int(jobs["w"].max()) if max_w is None else max_w
    ctx().global_batch(g.default_score(), to_dev(jobs), n, to_dev(codes), to_dev(nmask), mq, mt, mw, d_score,
                       d_cig, stride, d_nc, d_st)
    torch.cuda.synchronize()
    return (d_score.cpu().numpy(), d_cig.cpu().numpy().view(np.uint32).reshape(n, stride), d_nc.cpu().numpy(),
            d_st.cpu().numpy())


@pytest.mark.parametrize("seed,max_len", [(1, 160), (5, 300), (9, 40)])
def test_gpu_global_matches_oracle(seed, max_len):
    cj, u8 = nat.global_jobs(4000, seed, max_len=max_len)
    stride = int((cj["qlen"] + cj["tlen"]).max()) + 2
    s1, c1, n1, _ = nat.oracle_global(cj, u8, g.default_score(), stride)
    s2, c2, n2, st = run_global(gpu_jobs(cj), u8, stride)
    assert (st == 0).all(), np.unique(st)
    assert np.array_equal(s1, s2)
    assert np.array_equal(n1, n2)
    bad = [k for k in range(len(cj)) if not np.array_equal(c1[k, :n1[k]], c2[k, :n2[k]])]
    assert not bad, bad[:5]


def test_gpu_global_reversed_reads():
    """G3X_JOB_QREV/TREV read the planes backwards: the same as the oracle on reversed copies."""
    cj, u8 = nat.global_jobs(1500, 11)
    stride = int((cj["qlen"] + cj["tlen"]).max()) + 2
    rev = u8.copy()
    for j in cj:
        a, b = int(j["q_off"]), int(j["q_off"] + j["qlen"])
        rev[a:b] = u8[a:b][::-1]
        a, b = int(j["t_off"]), int(j["t_off"] + j["tlen"])
        rev[a:b] = u8[a:b][::-1]
    s1, c1, n1, _ = nat.oracle_global(cj, rev, g.default_score(), stride)
    s2, c2, n2, st = run_global(gpu_jobs(cj, g.JOB_QREV | g.JOB_TREV), u8, stride)
    assert (st == 0).all() and np.array_equal(s1, s2) and np.array_equal(n1, n2)
    assert all(np.array_equal(c1[k, :n1[k]], c2[k, :n2[k]]) for k in range(len(cj)))


def test_gpu_global_limits():
    """Jobs beyond the call's bounds, and CIGARs beyond the stride, get G3X_ERR_TOO_LONG."""
    cj, u8 = nat.global_jobs(600, 13, ws=(3, 5, 17))
    jobs = gpu_jobs(cj)
    stride = 4
    s1, c1, n1, _ = nat.oracle_global(cj, u8, g.default_score(), int((cj["qlen"] + cj["tlen"]).max()) + 2)
    s2, c2, n2, st = run_global(jobs, u8, stride, max_qlen=100, max_w=10)
    over = (cj["qlen"] > 100) | (cj["w"] > 10)
    assert (st[over] == g.G3X_ERR_TOO_LONG).all()
    fits = ~over & (n1 <= stride)
    assert (st[fits] == 0).all() and np.array_equal(s2[fits], s1[fits]) and np.array_equal(n2[fits], n1[fits])
    long_ = ~over & (n1 > stride)
    assert long_.any() and (st[long_] == g.G3X_ERR_TOO_LONG).all() and (n2[long_] == 0).all()


def test_gpu_global_nm_md():
    """NM and MD (the traceback stage's block after ksw_global2) equal the oracle's, itself
    pinned to the reference's own block (tests/test_global_oracle.py)."""
    import torch
    cj, u8 = nat.global_jobs(3000, 21, max_len=200)
    cj["flags"][::3] = g.JOB_MDRC
    jobs = gpu_jobs(cj)
    jobs["flags"] = cj["flags"]
    n = len(cj)
    stride = int((cj["qlen"] + cj["tlen"]).max()) + 2
    md_stride = 4 * stride + 16
    s1, c1, n1, _ = nat.oracle_global(cj, u8, g.default_score(), stride)
    nm1, md1 = nat.oracle_nm_md(cj, u8, c1, n1, md_stride)
    codes, nmask = g.pack_planes(u8)
    d_score = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_cig = torch.zeros(n * stride, dtype=torch.int32, device="cuda")
    d_nc = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_st = torch.full((n,), 99, dtype=torch.int32, device="cuda")
    d_nm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_md = torch.zeros(n * md_stride, dtype=torch.uint8, device="cuda")
    ctx().global_batch(g.default_score(), to_dev(jobs), n, to_dev(codes), to_dev(nmask), int(cj["qlen"].max()),
                       int(cj["tlen"].max()), int(cj["w"].max()), d_score, d_cig, stride, d_nc, d_st,
                       d_nm=d_nm, d_md=d_md, md_stride=md_stride)
    torch.cuda.synchronize()
    assert (d_st.cpu().numpy() == 0).all()
    assert np.array_equal(d_nm.cpu().numpy(), nm1)
    md = d_md.cpu().numpy().reshape(n, md_stride)
    md2 = [bytes(md[k]).split(b"\0")[0].decode() for k in range(n)]
    assert md2 == md1


@pytest.mark.parametrize("long_len", [0, 3500])
def test_gpu_global_both_ring_forms(long_len):
    """Short batches keep H and E as int16 pairs (-2^14 outside the band), batches with long
    sequences as int32 pairs (the reference's -2^30): both equal the oracle, scores from outside
    the band included (jobs whose band misses the last cell)."""
    cj, u8 = nat.global_jobs(1500, 21 + long_len, max_len=120, ws=(0, 1, 3, 10, 40))
    if long_len:
        rng = np.random.default_rng(long_len)
        extra = []
        for k in range(6):
            q = rng.integers(0, 4, long_len - 300 * k).astype(np.uint8)
            t = q.copy()
            t[rng.integers(0, len(t), 40)] = rng.integers(0, 4, 40)
            extra.append((q, t[: len(t) - 20 * k]))
        off = len(u8)
        ej = np.zeros(len(extra), cj.dtype)
        parts = [u8]
        for k, (q, t) in enumerate(extra):
            ej[k]["q_off"], ej[k]["t_off"], ej[k]["qlen"], ej[k]["tlen"], ej[k]["w"] = off, off + len(q), len(q), len(t), 60
            parts += [q, t]
            off += len(q) + len(t)
        cj, u8 = np.concatenate([cj, ej]), np.concatenate(parts)
    # a few jobs whose band cannot reach the last cell: query much longer than target + w
    out_of_band = (cj["qlen"] > cj["tlen"] + cj["w"])
    stride = int((cj["qlen"] + cj["tlen"]).max()) + 2
    s1, c1, n1, _ = nat.oracle_global(cj, u8, g.default_score(), stride)
    s2, c2, n2, st = run_global(gpu_jobs(cj), u8, stride)
    assert (st == 0).all(), np.unique(st)
    assert np.array_equal(s1, s2)
    assert np.array_equal(n1, n2)
    assert all(np.array_equal(c1[k, :n1[k]], c2[k, :n2[k]]) for k in range(len(cj)))
    assert out_of_band.any() and (s1[out_of_band] < -(1 << 29)).any()
