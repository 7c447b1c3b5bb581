"""The oracle's ksw_global2 (oracle/ksw_oracle.c) against the reference's own ksw_global2 with
push_cigar (bwa/src/ksw.cu:548, 694-809, compiled by oracle/build_ref.sh): equal scores on
every job, equal CIGARs wherever the reference's backtrack is defined (an in-band alignment
reaches the last cell)."""
import numpy as np
import pytest

import g3sa_b200 as g
from tests import native as nat


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_global_equals_reference(seed):
    jobs, u8 = nat.global_jobs(2500, seed)
    stride = int((jobs["qlen"] + jobs["tlen"]).max()) + 2
    sc = g.default_score()
    s1, c1, n1, cells = nat.oracle_global(jobs, u8, sc, stride)
    s2, c2, n2 = nat.ref_global(jobs, u8, sc, stride)
    assert np.array_equal(s1, s2)
    ok = s1 > nat.NEG_HALF
    assert ok.mean() > 0.5 and (~ok).any()
    assert np.array_equal(n1[ok], n2[ok])
    for k in np.nonzero(ok)[0]:
        assert np.array_equal(c1[k, :n1[k]], c2[k, :n2[k]]), k
    assert (n1[~ok] == 0).all()
    # CIGAR lengths add up to the sequences
    for k in np.nonzero(ok)[0][:300]:
        ops = c1[k, :n1[k]]
        ln, op = ops >> 4, ops & 0xF
        assert ln[op != 2].sum() == jobs["qlen"][k] and ln[op != 1].sum() == jobs["tlen"][k]


@pytest.mark.skipif(not nat.have_ref(), reason="oracle/_ref not built (no reference tree)")
@pytest.mark.parametrize("seed", [4, 5])
def test_oracle_nm_md_equals_reference(seed):
    jobs, u8 = nat.global_jobs(2000, seed)
    jobs["flags"][::3] = 4                      # the reverse-strand alphabet on a third of them
    stride = int((jobs["qlen"] + jobs["tlen"]).max()) + 2
    s, c, n, _ = nat.oracle_global(jobs, u8, g.default_score(), stride)
    md_stride = 4 * stride + 16
    nm1, md1 = nat.oracle_nm_md(jobs, u8, c, n, md_stride)
    nm2, md2 = nat.ref_nm_md(jobs, u8, c, n, md_stride)
    assert np.array_equal(nm1, nm2)
    assert md1 == md2
    assert any("^" in m for m in md1) and any(set("TGCA") & set(m) for m in md1) and (nm1 > 0).any()
