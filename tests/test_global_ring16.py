"""The premise of the global kernel's int16 ring (g3sa_b200/csrc/g3x_global.cu, Ring<true>):
when the batch's bound 2 max(o) + max(e) (qmax + tmax + 2) + max|mat| (min(qmax, tmax) + 1) is at
most 8000, running ksw_global2's recurrence (bwa/src/ksw.cu:706-779) with -2^14 outside the band
instead of -2^30 gives the same direction byte in every cell, stores only values that fit int16,
keeps every value inside the band above -2^13 and every value outside below it, and yields a
score that maps back to the -2^30 one by adding the same sum.  Checked here on the CPU, cell by
cell, on random pairs under random and extreme scorings up to the bound."""
import numpy as np
import pytest


def dp(q, t, mat, od, ed, oi, ei, w, neg):
    """ksw_global2's forward pass: (score, direction bytes, every stored H and E)."""
    qlen, tlen = len(q), len(t)
    H = np.full(qlen + 1, neg, np.int64)
    E = np.full(qlen + 1, neg, np.int64)
    H[0] = 0
    for j in range(1, min(qlen, w) + 1):
        H[j] = -(oi + ei * j)
    stored, dirs = [H.copy(), E.copy()], {}
    for i in range(tlen):
        beg, end = max(i - w, 0), min(i + w + 1, qlen)
        f = neg
        h1 = -(od + ed * (i + 1)) if beg == 0 else neg
        for j in range(beg, end):
            m = H[j] + mat[t[i] * 5 + q[j]]
            e = E[j]
            H[j] = h1
            d = 0 if m >= e else 1
            h = m if m >= e else e
            if h < f:
                d, h = 2, f
            h1 = h
            tt = m - od - ed
            e -= ed
            if e > tt:
                d |= 4
            else:
                e = tt
            E[j] = e
            tt = m - oi - ei
            f -= ei
            if f > tt:
                d |= 32
            else:
                f = tt
            dirs[i, j] = d
            stored += [np.array([H[j], E[j]])]
        if end <= qlen:
            H[end], E[end] = h1, neg
            stored += [np.array([h1, neg])]
    return int(H[qlen]), dirs, np.concatenate(stored)


def bound(od, ed, oi, ei, mat, qmax, tmax):
    return 2 * max(od, oi) + max(ed, ei) * (qmax + tmax + 2) + int(np.abs(mat).max()) * (min(qmax, tmax) + 1)


@pytest.mark.parametrize("seed", range(6))
def test_int16_ring_matches_int32(seed):
    rng = np.random.default_rng(1000 + seed)
    big = seed >= 3                  # scorings from the default to extreme ones inside the bound
    top, near = 0, False
    for it in range(40 if big else 25):
        qlen, tlen = int(rng.integers(0, 70 if big else 40)), int(rng.integers(0, 70 if big else 40))
        a = int(rng.integers(1, 40 if big else 3))
        b = int(rng.integers(1, 60 if big else 5))
        od, oi = (int(x) for x in rng.integers(0, 120 if big else 8, 2))
        ed, ei = (int(x) for x in rng.integers(1, 40 if big else 3, 2))
        if big and it == 0:          # close to the bound: 200 + 30 * 122 + 50 * 61 = 6910
            qlen, tlen, a, b, od, oi, ed, ei = 60, 60, 25, 50, 100, 100, 30, 30
        mat = np.full(25, -b, np.int64)
        for c in range(4):
            mat[c * 5 + c] = a
        mat[20:] = -1
        mat[4::5] = -1
        bd = bound(od, ed, oi, ei, mat, qlen, tlen)
        if bd > 8000:
            continue
        near = near or bd > 6000
        q = rng.integers(0, 5, qlen)
        t = q.copy() if rng.random() < 0.5 else rng.integers(0, 5, tlen)
        t = t[:tlen] if len(t) >= tlen else np.concatenate([t, rng.integers(0, 5, tlen - len(t))])
        w = int(rng.integers(0, 45))
        s32, d32, v32 = dp(q, t, mat, od, ed, oi, ei, w, -(1 << 30))
        s16, d16, v16 = dp(q, t, mat, od, ed, oi, ei, w, -(1 << 14))
        assert d16 == d32
        assert (v16 >= -(1 << 15)).all() and (v16 < (1 << 15)).all()          # int16 storage
        inside = v32 > -(1 << 29)
        assert (v16[inside] > -(1 << 13)).all() and (v16[~inside] < -(1 << 13)).all()
        assert (v16[~inside] - (-(1 << 14)) == v32[~inside] - (-(1 << 30))).all()
        finite = s16 > -(1 << 13)
        assert (s16 if finite else -(1 << 30) + (s16 + (1 << 14))) == s32
        top += 1
    assert top > 10 and (near or not big)
