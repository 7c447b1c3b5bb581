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
